/*
 * amss_b200.h -- C ABI of the B200-native AMSS-NCKU evolution hot path.
 *
 * Two layers:
 *
 * 1. Drop-in entry points with the reference's Fortran symbols and argument
 *    lists (gfortran "fortran3" mangling: lower case + trailing underscore,
 *    every argument by reference).  A caller linked against libamss_b200.so
 *    instead of the Fortran objects gets the same results computed on the
 *    GPU.  Arrays are host arrays in Fortran order (i fastest), exactly as the
 *    reference's Block::fgfs holds them; nothing is retained between calls.
 *
 * 2. The batched engine (amss_engine_*): blocks of every level stay resident
 *    in HBM, one kernel launch advances all blocks of a level by one RK4
 *    substep, and a whole step can be replayed as a CUDA graph.
 *
 * Return codes: 0 success; 1 NaN found in the input state (the reference's
 * `gont`); negative values are library errors (AMSS_ERR_*), with a message
 * available from amss_last_error().  There is no CPU fallback: without a
 * usable CUDA device every entry point fails with AMSS_ERR_NO_DEVICE.
 */
#ifndef AMSS_B200_H
#define AMSS_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define AMSS_OK 0
#define AMSS_NAN 1
#define AMSS_ERR_NO_DEVICE (-1)
#define AMSS_ERR_CUDA (-2)
#define AMSS_ERR_ARG (-3)
#define AMSS_ERR_UNSUPPORTED (-4)
#define AMSS_ERR_STATE (-5)

/* Last error message of the calling thread ("" if none). */
const char* amss_last_error(void);
/* Library version string. */
const char* amss_version(void);

/* ---------------------------------------------------------------------------
 * Drop-in per-block kernels
 * ------------------------------------------------------------------------- */

/* Replaces compute_rhs_bssn (bssn_rhs.f90:5-1184; C prototype bssn_rhs.h:37-54,
 * called per block from bssn_class.C:3059 and :3430).  GAUGE 0, Cell,
 * ghost_width 3.  Outputs: 24 RHS, 18 physical Christoffel symbols, 6 Ricci
 * components, and (co == 0) the 7 constraint residuals.  Returns 1 without
 * touching any output when the input state holds a NaN (bssn_rhs.f90:110-138). */
int compute_rhs_bssn_(
    int* ex, double* T, double* X, double* Y, double* Z,
    double* chi, double* trK, double* dxx, double* gxy, double* gxz, double* dyy, double* gyz, double* dzz,
    double* Axx, double* Axy, double* Axz, double* Ayy, double* Ayz, double* Azz,
    double* Gamx, double* Gamy, double* Gamz,
    double* Lap, double* betax, double* betay, double* betaz,
    double* dtSfx, double* dtSfy, double* dtSfz,
    double* chi_rhs, double* trK_rhs,
    double* gxx_rhs, double* gxy_rhs, double* gxz_rhs, double* gyy_rhs, double* gyz_rhs, double* gzz_rhs,
    double* Axx_rhs, double* Axy_rhs, double* Axz_rhs, double* Ayy_rhs, double* Ayz_rhs, double* Azz_rhs,
    double* Gamx_rhs, double* Gamy_rhs, double* Gamz_rhs,
    double* Lap_rhs, double* betax_rhs, double* betay_rhs, double* betaz_rhs,
    double* dtSfx_rhs, double* dtSfy_rhs, double* dtSfz_rhs,
    double* rho, double* Sx, double* Sy, double* Sz,
    double* Sxx, double* Sxy, double* Sxz, double* Syy, double* Syz, double* Szz,
    double* Gamxxx, double* Gamxxy, double* Gamxxz, double* Gamxyy, double* Gamxyz, double* Gamxzz,
    double* Gamyxx, double* Gamyxy, double* Gamyxz, double* Gamyyy, double* Gamyyz, double* Gamyzz,
    double* Gamzxx, double* Gamzxy, double* Gamzxz, double* Gamzyy, double* Gamzyz, double* Gamzzz,
    double* Rxx, double* Rxy, double* Rxz, double* Ryy, double* Ryz, double* Rzz,
    double* ham_Res, double* movx_Res, double* movy_Res, double* movz_Res,
    double* Gmx_Res, double* Gmy_Res, double* Gmz_Res,
    int* Symmetry, int* Lev, double* eps, int* co);

/* Replaces compute_rhs_Z4c (Z4c_rhs.f90:126-1295; C prototype bssn_rhs.h:142-160,
 * called per block from Z4c_class.C:207 and :575).  GAUGE 0, Cell, ghost_width 3,
 * kappa1 = 0.02, kappa2 = 0 (cpbc.f90:5-20).  State and RHS lists as
 * compute_rhs_bssn_ with Theta (TZ) after dtSfz.  The diagnostic outputs
 * (physical Christoffels, Ricci, the 7 constraint residuals) are always
 * computed, from the first 24 fields, as ricci_gamma and constraint_bssn do
 * (Z4c_rhs.f90:1266-1290); co is ignored.  Returns 1 without touching any
 * output when one of the 25 state fields holds a NaN (Z4c_rhs.f90:230-262). */
int compute_rhs_z4c_(
    int* ex, double* T, double* X, double* Y, double* Z,
    double* chi, double* trK, double* dxx, double* gxy, double* gxz, double* dyy, double* gyz, double* dzz,
    double* Axx, double* Axy, double* Axz, double* Ayy, double* Ayz, double* Azz,
    double* Gamx, double* Gamy, double* Gamz,
    double* Lap, double* betax, double* betay, double* betaz,
    double* dtSfx, double* dtSfy, double* dtSfz, double* TZ,
    double* chi_rhs, double* trK_rhs,
    double* gxx_rhs, double* gxy_rhs, double* gxz_rhs, double* gyy_rhs, double* gyz_rhs, double* gzz_rhs,
    double* Axx_rhs, double* Axy_rhs, double* Axz_rhs, double* Ayy_rhs, double* Ayz_rhs, double* Azz_rhs,
    double* Gamx_rhs, double* Gamy_rhs, double* Gamz_rhs,
    double* Lap_rhs, double* betax_rhs, double* betay_rhs, double* betaz_rhs,
    double* dtSfx_rhs, double* dtSfy_rhs, double* dtSfz_rhs, double* TZ_rhs,
    double* rho, double* Sx, double* Sy, double* Sz,
    double* Sxx, double* Sxy, double* Sxz, double* Syy, double* Syz, double* Szz,
    double* Gamxxx, double* Gamxxy, double* Gamxxz, double* Gamxyy, double* Gamxyz, double* Gamxzz,
    double* Gamyxx, double* Gamyxy, double* Gamyxz, double* Gamyyy, double* Gamyyz, double* Gamyzz,
    double* Gamzxx, double* Gamzxy, double* Gamzxz, double* Gamzyy, double* Gamzyz, double* Gamzzz,
    double* Rxx, double* Rxy, double* Rxz, double* Ryy, double* Ryz, double* Rzz,
    double* Hcon, double* Mxcon, double* Mycon, double* Mzcon,
    double* Gmxcon, double* Gmycon, double* Gmzcon,
    int* Symmetry, int* Lev, double* eps, int* co);

/* No counterpart in the reference.  compute_rhs_bssn_ for callers that cannot
 * allocate device memory (a host inside a memory pool it does not own, or one
 * whose device memory is reserved up front): same arguments, outputs and NaN
 * rule, but no cudaMalloc/cudaFree and no stream creation.  Its device staging
 * area is a static array of the library (23.4 MB per device) that every call
 * shares, so blocks are limited to AMSS_NOALLOC_MAX_POINTS points (and 4096
 * per extent; larger ones fail with AMSS_ERR_ARG), and calls that overlapped
 * on the GPU would race on it: the library serialises the calls of one
 * process with a lock held until each call's results are on the host.  Runs
 * on the per-thread default stream.  The first call on a device looks up the
 * array's address (again after a device reset) and, under CUDA's default lazy
 * module loading, loads the library's device code, which is when the array's
 * memory is taken: make that first call before reserving the rest of the
 * device's memory, and outside any stream capture. */
#define AMSS_NOALLOC_MAX_POINTS 32768
int amss_compute_rhs_bssn_noalloc(
    int* ex, double* T, double* X, double* Y, double* Z,
    double* chi, double* trK, double* dxx, double* gxy, double* gxz, double* dyy, double* gyz, double* dzz,
    double* Axx, double* Axy, double* Axz, double* Ayy, double* Ayz, double* Azz,
    double* Gamx, double* Gamy, double* Gamz,
    double* Lap, double* betax, double* betay, double* betaz,
    double* dtSfx, double* dtSfy, double* dtSfz,
    double* chi_rhs, double* trK_rhs,
    double* gxx_rhs, double* gxy_rhs, double* gxz_rhs, double* gyy_rhs, double* gyz_rhs, double* gzz_rhs,
    double* Axx_rhs, double* Axy_rhs, double* Axz_rhs, double* Ayy_rhs, double* Ayz_rhs, double* Azz_rhs,
    double* Gamx_rhs, double* Gamy_rhs, double* Gamz_rhs,
    double* Lap_rhs, double* betax_rhs, double* betay_rhs, double* betaz_rhs,
    double* dtSfx_rhs, double* dtSfy_rhs, double* dtSfz_rhs,
    double* rho, double* Sx, double* Sy, double* Sz,
    double* Sxx, double* Sxy, double* Sxz, double* Syy, double* Syz, double* Szz,
    double* Gamxxx, double* Gamxxy, double* Gamxxz, double* Gamxyy, double* Gamxyz, double* Gamxzz,
    double* Gamyxx, double* Gamyxy, double* Gamyxz, double* Gamyyy, double* Gamyyz, double* Gamyzz,
    double* Gamzxx, double* Gamzxy, double* Gamzxz, double* Gamzyy, double* Gamzyz, double* Gamzzz,
    double* Rxx, double* Rxy, double* Rxz, double* Ryy, double* Ryz, double* Rzz,
    double* ham_Res, double* movx_Res, double* movy_Res, double* movz_Res,
    double* Gmx_Res, double* Gmy_Res, double* Gmz_Res,
    int* Symmetry, int* Lev, double* eps, int* co);

/* Replaces rungekutta4_rout (rungekutta4_rout.f90:94-139; rungekutta4_rout.h:34-38,
 * called per field from bssn_class.C:3119 and :3430-3525).  RK4 = 0..3. */
int rungekutta4_rout_(int* ex, double* dT, double* f0, double* f1, double* f_rhs, int* RK4);

/* Replaces sommerfeld_routbam (sommerfeld_rout.f90:223-449; sommerfeld_rout.h:33-37,
 * called per field on level 0 from bssn_class.C:3109). */
void sommerfeld_routbam_(int* ex, double* X, double* Y, double* Z,
                         double* xmin, double* ymin, double* zmin, double* xmax, double* ymax, double* zmax,
                         double* f_rhs, double* f0, double* velocity, double* SoA, int* Symmetry);

/* Replaces sommerfeld_rout (sommerfeld_rout.f90:9-221; sommerfeld_rout.h:26-30,
 * called per field on levels > 0 from bssn_class.C:3127).  Only precor == 1,
 * the branch on the evolution path (copy f0 onto the patch faces), is
 * implemented; other values fail with AMSS_ERR_UNSUPPORTED. */
void sommerfeld_rout_(int* ex, double* X, double* Y, double* Z,
                      double* xmin, double* ymin, double* zmin, double* xmax, double* ymax, double* zmax,
                      double* dT, double* chi0, double* Lap0, double* f0, double* f, double* SoA,
                      int* Symmetry, int* precor);

/* Replaces enforce_ga (enforce_algebra.f90:72-133; enforce_algebra.h:26-28,
 * called from bssn_class.C:3052 and :3416). In place. */
void enforce_ga_(int* ex, double* dxx, double* gxy, double* gxz, double* dyy, double* gyz, double* dzz,
                 double* Axx, double* Axy, double* Axz, double* Ayy, double* Ayz, double* Azz);

/* Replaces lowerboundset (fmisc.f90:1644-1657; fmisc.h:210, called from
 * bssn_class.C:3156 and :3525). In place. */
void lowerboundset_(int* ex, double* chi, double* tinny);

/* Replaces get_lousto_nbhs (initial_puncture.f90:1970-2202; C prototype
 * initial_puncture.h:165-174, called per block from bssn_class.C:1165):
 * Lousto's approximate puncture data for N punctures (Mass[N], Porg/Pmom/Spin
 * [3N]; zero momenta and spins give Brill-Lindquist), stored as offsets
 * (chi - 1, Lap - 1; metric offsets, trK, Gam, beta, dtSf zero).  The reference
 * prototype returns void; this one returns 0 or an AMSS_ERR_* code, which a
 * caller using the void prototype may ignore.  At most 16 punctures. */
int get_lousto_nbhs_(int* ex, double* X, double* Y, double* Z, double* chi, double* trK,
                     double* gxx, double* gxy, double* gxz, double* gyy, double* gyz, double* gzz,
                     double* Axx, double* Axy, double* Axz, double* Ayy, double* Ayz, double* Azz,
                     double* Gmx, double* Gmy, double* Gmz, double* Lap, double* Sfx, double* Sfy, double* Sfz,
                     double* dtSfx, double* dtSfy, double* dtSfz, double* Mass, double* Porg, double* Pmom,
                     double* Spin, int* N);

/* No counterpart in the reference.  The vector-Jacobian product of
 * get_lousto_nbhs_ with zero momenta and spins (Brill-Lindquist) with respect
 * to the masses and positions: given the adjoints chi_b, lap_b of the chi and
 * Lap outputs (host, Fortran order), dMass[N] and dPorg[3N].  The other outputs
 * do not depend on them in this case. */
int amss_lousto_vjp(const int* ex, const double* X, const double* Y, const double* Z, int N, const double* Mass,
                    const double* Porg, const double* chi_b, const double* lap_b, double* dMass, double* dPorg);

/* ---------------------------------------------------------------------------
 * Batched engine: device-resident blocks, one launch per level substep.
 * ------------------------------------------------------------------------- */

typedef struct amss_engine amss_engine;

typedef struct {
  int precision;      /* 0: FP64; 1: mixed (FP32 stencils/stages, FP64 state and accumulator) */
  int symmetry;       /* 0 none, 1 equatorial, 2 octant (ABE::Symmetry) */
  double eps;         /* KO dissipation (ABE::... dissipation) */
  double chitiny;     /* chi floor as the reference stores it: BSSN::chitiny - 1 */
  int kernel;         /* 0: split substep (stencil pass + pointwise pass, default); 1: fused single pass */
  int formulation;    /* 0: BSSN, 24 fields (bssn_rhs.f90); 1: Z4c, 25 fields with Theta last
                         (Z4c_rhs.f90:126-1295, ABEtype 2); Z4c needs kernel 0 */
} amss_params;

/* Create an engine on the current CUDA device.  Returns NULL on failure. */
amss_engine* amss_engine_create(const amss_params* prm);
void amss_engine_destroy(amss_engine* e);

/* Add one block of `level`: ex points per direction, its cell-centred bbox
 * (Block::bbox, coordinates X[j] = bbox_lo + (j + 0.5) h) and the bbox of the
 * patch it belongs to (decides which faces take the outer boundary rule).
 * Returns the block id (>= 0) or an error code. */
int amss_engine_add_block(amss_engine* e, int level, const int ex[3], const double bbox[6],
                          const double patch_bbox[6]);

/* Allocate HBM for all blocks and build the per-level work lists. */
int amss_engine_commit(amss_engine* e);

/* Copy one block's 24-field state (host, Fortran order, field-major) in/out. */
int amss_engine_set_state(amss_engine* e, int block, const double* host_state);
int amss_engine_get_state(amss_engine* e, int block, double* host_state);
/* A block's state `back` level steps before the current one (back 0..2; 0 is
 * amss_engine_set/get_state), for checkpoints (checkpoint::writecheck_cgh
 * stores StateList and OldStateList, checkpoint.C:132-190, bssn_class.C:682-683)
 * and regrids. */
int amss_engine_set_time_level(amss_engine* e, int block, int back, const double* host_state);
int amss_engine_get_time_level(amss_engine* e, int block, int back, double* host_state);
/* Steps a level has taken (the time interpolation of its children is quadratic
 * from the second step on), and setting it when a run resumes from a checkpoint. */
int amss_engine_level_clock(amss_engine* e, int level, int* steps);
int amss_engine_set_level_clock(amss_engine* e, int level, int steps);
/* Device pointer of field 0 of a block's state and the field stride in elements. */
int amss_engine_state_device(amss_engine* e, int block, double** dptr, long long* field_stride);

/* AMR hierarchies: the grid origin (coordinate of the lower face of global
 * cell 0 on every level) and the level-0 cell size; level l has cell size
 * h0 / 2^l and coarse cell k has the fine children 2k, 2k+1. */
int amss_engine_set_grid(amss_engine* e, const double x0[3], double h0);

/* Add one block of an AMR level.  org: global level index of array element 0;
 * ex: array extent; [own_lo, own_hi): the cells the block owns (the rest of its
 * array are ghost cells, ghost_width 3, filled from their owners after every
 * substep as Parallel::Sync does); [phys_lo, phys_hi): the physical box of the
 * block's patch, which on levels > 0 is surrounded by `buffer` cells
 * (buffer_width 6) filled by prolongation from the parent level after each step
 * (Parallel::OutBdLow2Hi).  `patch` identifies the patch within its level.
 * Returns the block id or an error code. */
int amss_engine_add_amr_block(amss_engine* e, int level, int patch, const int org[3], const int ex[3],
                              const int own_lo[3], const int own_hi[3], const int phys_lo[3],
                              const int phys_hi[3], int buffer);

/* One Berger-Oliger coarse step of the whole hierarchy (bssn_class::RecursiveStep,
 * bssn_class.C:2323-2414, with RPS 1 and time refinement from level 1): level l
 * takes 2^l RK4 steps of dt0 / 2^l, each followed by restriction into and
 * prolongation from its parent (bssn_class::RestrictProlong, :5724-5903) with
 * quadratic time interpolation of the parent at intermediate times. */
int amss_engine_coarse_step(amss_engine* e, double dt0);

/* Capture `nsteps` coarse steps as one CUDA graph and replay it `replays` times. */
int amss_engine_run_coarse_graph(amss_engine* e, double dt0, int nsteps, int replays);

/* Points (array cells of all blocks) of a level. */
long long amss_engine_level_points(amss_engine* e, int level);

/* Apply enforce_ga to every block's state once (the reference does this at
 * the start of every step; the engine then keeps states in that form). */
int amss_engine_enforce(amss_engine* e);

/* Advance every block of `level` by one RK4 step of size dt on the engine's
 * stream (asynchronous).  Single-level hierarchies only in this form. */
int amss_engine_step_level(amss_engine* e, int level, double dt);

/* Capture `nsteps` calls of amss_engine_step_level(level, dt) as one CUDA
 * graph and replay it `replays` times. */
int amss_engine_run_graph(amss_engine* e, int level, double dt, int nsteps, int replays);

/* No counterpart in the reference (its work split is the MPI block layout).
 * Tiling of the stencil pass of one level, the knob amss_b200.autotune
 * searches: x-y tile width (8..64 columns, H = 256 / width rows; 0 restores
 * the default, the block's x extent cut into pieces of at most 64) and the
 * number of z-slabs each block's march is cut into (1..16; slabs are at least
 * 8 planes).  Results do not depend on it.  Waits for the engine's stream;
 * not inside a stream capture. */
int amss_engine_set_level_tiling(amss_engine* e, int level, int tile_w, int zsplit);
/* The level's tiling (as set; 0 = default width) and its stencil work items. */
int amss_engine_get_level_tiling(amss_engine* e, int level, int* tile_w, int* zsplit, int* nitems);
/* No reference counterpart: which compiled form of the stencil pass a level
 * uses, 0 (two resident CTAs per SM, the default) or 1 (four in FP64, three in
 * FP32, fewer registers with some spills).  Results do not depend on it. */
int amss_engine_set_level_occupancy(amss_engine* e, int level, int occ);
int amss_engine_get_level_occupancy(amss_engine* e, int level, int* occ);
/* No reference counterpart: the cells a coarse step's final RK4 substep
 * updates on a level.  In a coarse step (amss_engine_coarse_step and its
 * graph) every step of a refined level is followed by RestrictProlong
 * (bssn_class.C:5724-5903), whose prolongation overwrites the level's buffer
 * cells; the restriction before it reads the new state at most 2 cells past
 * the physical box (restrict3), and the finer levels' prolongation reads it
 * around their patches.  Where commit finds every such read within `pad` = 2
 * cells of the owning block's physical box and every buffer cell prolonged,
 * the final substep updates only each owned block's cells within that
 * distance; the other cells' new values would be overwritten unread, so the
 * coarse step's results are the same bit for bit.  *pad = -1: no such
 * regions (level 0, or a hierarchy that fails the test).  A single level step
 * (amss_engine_step_level) never uses them.  Every substep (the final one
 * too, where it has no regions) skips a block's ghost cells when commit finds
 * that the same-level sync after it overwrites every ghost cell of the level.
 * *points: the cells a coarse step's final substep updates on this rank's
 * blocks of the level. */
int amss_engine_level_final_region(amss_engine* e, int level, int* pad, long long* points);

/* Moving-box regrid (cgh::Regrid_Onelevel, cgh.C:1304-1506, whose data step is
 * cgh::recompose_cgh_Onelevel and Parallel::fill_level_data, Parallel.C).
 * `dst` is a committed engine over the new hierarchy (same grid, fields and
 * precision), `src` the engine it replaces, both at the same time.  For one
 * level and one time level (back 0: the current state; 1: the one a level
 * step before), every cell of dst's blocks (ghosts included) that a block of
 * src's level owns is copied, and every cell outside all of src's patches
 * (their buffers included) is prolonged (prolong3) from src's parent level:
 * from its current state for back 0, from its state interpolated in time to
 * the midpoint of its current and previous levels (average2, Parallel.C
 * :4383-4441) for back 1, which overwrites the parent's accumulators.  The
 * level's clock (ring index, steps taken) is copied too.  A cell outside the
 * old parent's blocks (boxes not nested) fails with AMSS_ERR_ARG. */
int amss_engine_regrid_fill(amss_engine* dst, amss_engine* src, int level, int back);

/* Wait for the engine's stream; returns 1 if any substep saw a NaN, else 0. */
int amss_engine_sync(amss_engine* e);

/* The engine's CUDA stream (cudaStream_t), for timing with events. */
void* amss_engine_stream(amss_engine* e);

/* Number of kernel launches the engine issued so far. */
long long amss_engine_launch_count(amss_engine* e);

/* The constraint monitor of one level (bssn_class.C:7463-7484,
 * Z4c_class.C:2491-2510, with Parallel::L2Norm, Parallel.C:4214-4243, and
 * l2normhelper, fmisc.f90:1263-1309): norms[0..6] = sqrt(sum c^2 dx dy dz) of
 * the Hamiltonian, the 3 momentum and the 3 Gamma constraints (compute_rhs_bssn
 * with co = 0, bssn_rhs.f90:1044-1135; constraint_bssn for Z4c) of the level's
 * current state, norms[7] that of Theta (Z4c; 0 for BSSN), in FP64 whatever
 * the engine's precision.  Cells: a block added by bbox contributes
 * its array less 3 ghost cells on each side whose outer cell is not within one
 * cell of its patch box; an AMR block its owned cells inside its patch,
 * buffer cells included.  Waits for the engine's stream. */
int amss_engine_constraint_norms(amss_engine* e, int level, double norms[8]);
/* The same norms over the level's first patch only, as the reference's
 * Constraint_Out takes them (Parallel::L2Norm(GH->PatL[lev]->data, ...),
 * bssn_class.C:7475): the first block's patch, or for blocks added by bbox
 * those sharing its patch box.  Equal to amss_engine_constraint_norms on a
 * level of one patch. */
int amss_engine_constraint_norms_first_patch(amss_engine* e, int level, double norms[8]);

/* Values of fields at points of one level (Parallel::PatList_Interp_Points,
 * Parallel.C:5614-5667, with Patch::Interp_Points, MPatch.C:339-500, and
 * global_interp, fmisc.f90:712-794: 6-point Lagrange per axis by Neville's
 * scheme, z then y then x, mirrored cells times the field's parity at a
 * symmetry plane).  xyz: npts points (x, y, z); fields: nvar state indices;
 * soa: 3 parities per field (NULL: all +1); out: npts x nvar.  found[p]
 * (may be NULL) is 0 when no patch of the level holds point p -- the
 * reference's `false`, on which compute_Porg_rhs (bssn_class.C:6879-6932)
 * tries the next coarser level -- and its values are 0.  A point inside a
 * patch but in none of its blocks, or a stencil that leaves its block, is
 * AMSS_ERR_ARG.  Reads the current state; waits for the engine's stream. */
int amss_engine_interp_points(amss_engine* e, int level, int npts, const double* xyz, int nvar, const int* fields,
                              const double* soa, double* out, int* found);

/* Puncture tracking (bssn_class::Step with MAPBH 0: bssn_class.C:3360-3390,
 * :3730-3760, :3804-3812, :3890-3898; compute_Porg_rhs, :6879-6932;
 * rungekutta4_scalar, rungekutta4_rout.f90:6-47).  n <= 10 positions
 * (x, y, z) = Porg0; from then on every step of the finest level also
 * advances them on the device: at each RK4 substep minus the shift of the
 * substep's input state, interpolated as amss_engine_interp_points does,
 * drives a scalar RK4 (|z| kept with Symmetry > 0, |x|, |y| with Symmetry 2).
 * The mixed form reads the shift of its FP32 stages; n = 0 stops tracking.
 * The reference tries coarser levels when a puncture leaves the finest one;
 * the engine flags it instead, and amss_engine_get_punctures then fails with
 * AMSS_ERR_STATE. */
int amss_engine_set_punctures(amss_engine* e, int n, const double* pos);

/* The tracked positions (3 n doubles) after the steps issued so far; waits
 * for the engine's stream. */
int amss_engine_get_punctures(amss_engine* e, double* pos);

/* ---- Wave extraction (bssn_class::AnalysisStuff, bssn_class.C:6945-7285).
 *
 * amss_engine_psi4: bssn_class::Compute_Psi4 (bssn_class.C:6210-6298) with
 * getnp4 (getnp4.f90:12-452; Psi4type 0, tetradtype 2): the Newman-Penrose
 * scalar Psi4 of the level's current state on every point of its blocks,
 * then the level's ghost sync.  The Christoffel symbols and Ricci tensor it
 * needs are those of the same state (the reference reuses the last
 * compute_rhs_bssn outputs of the level).  The result lives in each block's
 * RK4 accumulator, fields 0 (Rpsi4) and 1 (Ipsi4), until the next step;
 * amss_engine_get_psi4 copies a block's two fields to the host (2 x npts).
 * A Z4c engine takes them from its first 24 fields, as Z4c_class inherits
 * Compute_Psi4 (its Christoffel and Ricci outputs are ricci_gamma's, the
 * BSSN formulas).
 *
 * amss_engine_psi4_modes: surface_integral::surf_Wave (surface_integral.C:
 * 197-377 with GaussInt; its sphere, :39-181): Psi4 interpolated on the
 * sphere of radius rex (N_theta = 2 nquarter Gauss-Legendre nodes in
 * cos(theta), N_phi = 4 nquarter midpoints in phi, reduced per symmetry) and
 * projected on the spin-weight -2 harmonics: RP, IP get (maxl+1)^2 - 4 values,
 * l = 2..maxl, m = -l..l, the bssn_psi4.dat columns.  Every sphere point must
 * lie in the level's patches (AMSS_ERR_ARG otherwise). */
int amss_engine_psi4(amss_engine* e, int level);
int amss_engine_get_psi4(amss_engine* e, int block, double* host);
int amss_engine_psi4_modes(amss_engine* e, int level, double rex, int nquarter, int maxl, double* RP, double* IP);

/* surface_integral::surf_MassPAng (surface_integral.C:2247-2512, GaussInt,
 * with admmass_bssn, fadmquantites_bssn.f90:5-65): the ADM mass, linear
 * momentum and angular momentum through the sphere of radius rex of the same
 * quadrature, from the level's current state.  out[7]: mass, Px, Py, Pz, Sx,
 * Sy, Sz, the bssn_ADMQs.dat columns (Symmetry 1 gives only Px, Py, Sz of the
 * momenta, Symmetry 2 none; the others are 0).  Overwrites accumulator
 * fields 2-4 (Psi4 in fields 0, 1 stays). */
int amss_engine_adm_integrals(amss_engine* e, int level, double rex, int nquarter, double out[7]);

/* ---- Blocks divided among ranks, one engine per GPU (Parallel::distribute,
 * Parallel.C:504-827, assigns the reference's blocks to MPI ranks;
 * Parallel::Sync / transfer, Parallel.C:3677-3776 and :3508-3592, move the
 * ghost, restriction and prolongation segments between them).
 *
 * Every rank builds the same hierarchy (same blocks in the same order) and
 * names the owner of each block before amss_engine_commit; an engine then
 * allocates and steps only its own blocks.  Each transfer (the ghost sync of
 * a level after every substep and step, the restriction into and the
 * prolongation from the parent after a fine step) runs on the rank that owns
 * the source block, into the destination block or, when another rank owns
 * that, into a staging region that the exchange delivers and the receiver
 * copies in.  The results are those of one engine holding every block, bit
 * for bit.  A rank engine refuses what needs the whole hierarchy
 * (graph capture, puncture tracking, point interpolation, regrid) with
 * AMSS_ERR_UNSUPPORTED; its constraint sums cover its own blocks. */

/* Before commit: this engine is `rank` of `nranks` (default 0 of 1), then
 * the owner of each block (default 0). */
int amss_engine_set_rank(amss_engine* e, int rank, int nranks);
int amss_engine_set_block_owner(amss_engine* e, int block, int owner);

/* Transport 1, ranks in one process (one host thread per rank, each with its
 * engine's device current): create a group of nranks, join every committed
 * rank engine, then step all ranks concurrently.  At each exchange the ranks
 * meet at a host barrier; one that does not arrive within timeout_s seconds
 * fails every rank's step with AMSS_ERR_STATE and the group stays failed.
 * Destroy the engines before the group. */
typedef struct amss_group amss_group;
amss_group* amss_group_create(int nranks, double timeout_s);
void amss_group_destroy(amss_group* g);
int amss_group_join(amss_engine* e, amss_group* g);
int amss_group_barrier(amss_group* g);   /* the exchange's host barrier alone */

/* Transport 2, NCCL (one process per GPU): rank 0 makes a unique id (128
 * bytes), the caller broadcasts it, every rank passes it after commit
 * (collective, ncclCommInitRank).  The exchange is a grouped ncclSend /
 * ncclRecv on the engine's stream.  libnccl.so.2 is opened at run time. */
int amss_nccl_unique_id(unsigned char id[128]);
int amss_engine_set_nccl(amss_engine* e, const unsigned char id[128]);

/* The unsquared sums behind amss_engine_constraint_norms (whose values are
 * their square roots) over this engine's blocks: the ranks add them up. */
int amss_engine_constraint_sums(amss_engine* e, int level, double sums[8]);

/* Transfer plans without a device (for checking a partition on any host):
 * amss_plan_create takes the parameters of amss_engine_create; add blocks,
 * ranks and owners as for an engine, then amss_plan_commit.  The plan
 * queries below work on plans and committed engines alike. */
amss_engine* amss_plan_create(const amss_params* prm);
int amss_plan_commit(amss_engine* e);
int amss_engine_xfer_count(amss_engine* e);
/* info: kind (0 ghost sync, 1 restriction, 2 prolongation), level (the fine
 * level for 1 and 2), boxes over all ranks, boxes crossing ranks, run boxes,
 * unpack boxes, staging-out bytes, staging-in bytes. */
int amss_engine_xfer_info(amss_engine* e, int xfer, long long info[8]);
/* list 0: the boxes this rank's transfer kernel computes; 1: the copies from
 * received staging blocks.  8 ints per box: dst, src, lo[3], n[3]; block ids
 * past the hierarchy's are staging blocks.  out NULL: the count. */
int amss_engine_xfer_boxes(amss_engine* e, int xfer, int list, int* out, int cap);
/* dir 0: send, 1: receive; 3 values per peer: rank, byte offset, bytes. */
int amss_engine_xfer_peers(amss_engine* e, int xfer, int dir, long long* out, int cap);
/* A staging block: org[3], ex[3], byte offset, arena (0 out, 1 in).  Its
 * buffers start at the offset: nf FP64 fields of ex points, or the stage
 * fields (FP32 in the mixed form, then 5 FP64 side fields 256-byte aligned). */
int amss_engine_staging_block(amss_engine* e, int id, long long out[8]);

/* ---- Adjoint of a single-patch BSSN evolution (no reference counterpart:
 * the reference has no derivative code; the forward it differentiates is the
 * level-0 RK4 step of bssn_class::Step, bssn_class.C:2981-3700, with
 * enforce_ga, lowerboundset and the Sommerfeld outer boundary).
 *
 * One block of ex points per direction on its cell-centred bbox, FP64,
 * GAUGE 0, no symmetry.  The loss is L = sum over the cells at least 3 cells
 * from every face of H^2 dx dy dz, H the Hamiltonian constraint of the final
 * state.  The gradient is dL/d(initial state) (24 fields, field-major, the
 * same host layout as amss_engine_set_state), computed by reverse-mode over
 * RK4 with a checkpoint every `ck` steps: every segment but the last is recomputed
 * once; the forward keeps the last segment's stages, and, where the device has room,
 * every substep's stencil terms of a segment (4 ck x 135 fields). */
typedef struct amss_adjoint amss_adjoint;

/* chitiny: the lowerboundset floor on chi (bssn_class.C:179, :3156).  NULL on failure. */
amss_adjoint* amss_adjoint_create(const int ex[3], const double bbox[6], double eps, double chitiny);
void amss_adjoint_destroy(amss_adjoint* a);
int amss_adjoint_set_state(amss_adjoint* a, const double* host_state);
int amss_adjoint_get_state(amss_adjoint* a, double* host_state);
/* nsteps RK4 steps of dt from the state set; *loss = L of the final state. */
int amss_adjoint_forward(amss_adjoint* a, double dt, int nsteps, int ck, double* loss);
/* dL/d(state before the last amss_adjoint_forward) into host_grad (24 fields). */
int amss_adjoint_backward(amss_adjoint* a, double* host_grad);
void* amss_adjoint_stream(amss_adjoint* a);
long long amss_adjoint_launch_count(amss_adjoint* a);

#ifdef __cplusplus
}
#endif

#endif /* AMSS_B200_H */
