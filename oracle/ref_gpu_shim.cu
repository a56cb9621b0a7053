// ref_gpu_shim.cu -- C entry into the reference's 2015 CUDA port of
// compute_rhs_bssn (gpu_rhs, bssn_gpu.cu:1985; prototype bssn_gpu.h:26),
// compiled together with that file by oracle/build_ref.py into
// oracle/_ref/libref_bssn_gpu.so.
//
// TEST INFRASTRUCTURE ONLY: a second, independent statement of the reference's
// right-hand side that the oracle is checked against; nothing in the product
// loads it.
//
// gpu_rhs takes its scalars by C++ reference; this shim gives ctypes a plain
// extern "C" symbol with pointers in the same order (after gpu_rhs's
// `calledby`, which selects the outputs it copies back), and supplies the
// reference's result-dump hook compare_result (bssn_macro.h:90, defined in
// bssn_macro.C:78 against Fortran dump files the reference does not ship),
// which gpu_rhs only calls under RESULT_CHECK.
#include "bssn_gpu.h"

int compare_result(int, double*, int) { return 0; }

extern "C" int ref_gpu_rhs(
    int calledby, int* ex, double* T, double* X, double* Y, double* Z, double* chi, double* trK, double* dxx, double* gxy,
    double* gxz, double* dyy, double* gyz, double* dzz, double* Axx, double* Axy, double* Axz, double* Ayy,
    double* Ayz, double* Azz, double* Gamx, double* Gamy, double* Gamz, double* Lap, double* betax, double* betay,
    double* betaz, double* dtSfx, double* dtSfy, double* dtSfz, double* chi_rhs, double* trK_rhs, double* gxx_rhs,
    double* gxy_rhs, double* gxz_rhs, double* gyy_rhs, double* gyz_rhs, double* gzz_rhs, double* Axx_rhs,
    double* Axy_rhs, double* Axz_rhs, double* Ayy_rhs, double* Ayz_rhs, double* Azz_rhs, double* Gamx_rhs,
    double* Gamy_rhs, double* Gamz_rhs, double* Lap_rhs, double* betax_rhs, double* betay_rhs, double* betaz_rhs,
    double* dtSfx_rhs, double* dtSfy_rhs, double* dtSfz_rhs, double* rho, double* Sx, double* Sy, double* Sz,
    double* Sxx, double* Sxy, double* Sxz, double* Syy, double* Syz, double* Szz, double* Gamxxx, double* Gamxxy,
    double* Gamxxz, double* Gamxyy, double* Gamxyz, double* Gamxzz, double* Gamyxx, double* Gamyxy, double* Gamyxz,
    double* Gamyyy, double* Gamyyz, double* Gamyzz, double* Gamzxx, double* Gamzxy, double* Gamzxz, double* Gamzyy,
    double* Gamzyz, double* Gamzzz, double* Rxx, double* Rxy, double* Rxz, double* Ryy, double* Ryz, double* Rzz,
    double* ham_Res, double* movx_Res, double* movy_Res, double* movz_Res, double* Gmx_Res, double* Gmy_Res,
    double* Gmz_Res, int* Symmetry, int* Lev, double* eps, int* co) {
  // calledby (bssn_macro.h:69-70): 0, CALLED_BY_STEP, copies the right-hand sides back;
  // 1, CALLED_BY_CONSTRAINT, the Christoffel symbols, Ricci components and residuals
  return gpu_rhs(calledby, 0, ex, *T, X, Y, Z, chi, trK, dxx, gxy, gxz, dyy, gyz, dzz, Axx, Axy, Axz, Ayy, Ayz, Azz,
                 Gamx, Gamy, Gamz, Lap, betax, betay, betaz, dtSfx, dtSfy, dtSfz, chi_rhs, trK_rhs, gxx_rhs,
                 gxy_rhs, gxz_rhs, gyy_rhs, gyz_rhs, gzz_rhs, Axx_rhs, Axy_rhs, Axz_rhs, Ayy_rhs, Ayz_rhs,
                 Azz_rhs, Gamx_rhs, Gamy_rhs, Gamz_rhs, Lap_rhs, betax_rhs, betay_rhs, betaz_rhs, dtSfx_rhs,
                 dtSfy_rhs, dtSfz_rhs, rho, Sx, Sy, Sz, Sxx, Sxy, Sxz, Syy, Syz, Szz, Gamxxx, Gamxxy, Gamxxz,
                 Gamxyy, Gamxyz, Gamxzz, Gamyxx, Gamyxy, Gamyxz, Gamyyy, Gamyyz, Gamyzz, Gamzxx, Gamzxy, Gamzxz,
                 Gamzyy, Gamzyz, Gamzzz, Rxx, Rxy, Rxz, Ryy, Ryz, Rzz, ham_Res, movx_Res, movy_Res, movz_Res,
                 Gmx_Res, Gmy_Res, Gmz_Res, *Symmetry, *Lev, *eps, *co);
}
