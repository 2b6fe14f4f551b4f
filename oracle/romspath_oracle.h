/*
 * romspath_oracle.h -- CPU FP64 restatement of the ROMSPath per-particle
 * time step (TEST INFRASTRUCTURE ONLY).
 *
 * This oracle is the checker for the CUDA path in romspath_b200/.  Only the
 * tests, the smoke check and the CPU-baseline leg of the benchmark may load
 * it; the product never routes through it.
 *
 * PARITY STATUS: parity unpinned against the reference binary.  The
 * reference is Fortran 90 + NetCDF and ships no tests, no golden vectors and
 * no known-answer files; no Fortran compiler exists here, so it cannot be
 * built and run.  The restatement is line-faithful to the reference source
 * (each function cites the file:line it follows) and is pinned only by
 * (a) the published MT19937 known answers (identical to C++ std::mt19937),
 * (b) analytic invariants (polintd exact on quadratics, s-level formulas,
 *     bilinear exactness, reflection symmetry, smoothing-spline limits).
 *
 * Conventions: every 2-D/3-D array is Fortran column-major with 1-based
 * index semantics, exactly as the reference's GRIDS(ng) / HYDRODATA(ng)
 * arrays: H(xi_rho,eta_rho), U(xi_u,eta_u,N), V(xi_v,eta_v,N),
 * W(xi_rho,eta_rho,N+1), AKs(xi_rho,eta_rho,N+1), zeta(xi_rho,eta_rho).
 * xi_u = xi_rho-1, eta_u = eta_rho, xi_v = xi_rho, eta_v = eta_rho-1.
 *
 * Arithmetic: plain IEEE FP64, no FMA contraction (-ffp-contract=off), the
 * reference's left-to-right evaluation order.
 */
#ifndef ROMSPATH_ORACLE_H
#define ROMSPATH_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_MAXNGRID 5

/* Per-particle flag bits (documented deviations where the reference is
 * undefined).  Identical values are used by the CUDA path. */
#define ORC_FLAG_OOB        0x01u /* a gather index left its array; clamped */
#define ORC_FLAG_NODE       0x02u /* getcoeff at an exact node (0/0 pinned)   */
#define ORC_FLAG_WBOT       0x04u /* w-level walk below level 1 (reads s_w(0)) */
#define ORC_FLAG_WTOP       0x08u /* w-level walk above level N+1            */
#define ORC_FLAG_SPLINE     0x10u /* smooth() secant iteration cap reached    */

typedef struct {
    int xi_rho, eta_rho, N;      /* N = s_rho; s_w = N+1 */
    int vtransform;
    double hc;
    const double *h, *pm, *pn;   /* (xi_rho, eta_rho) */
    const int32_t *mask_rho;     /* (xi_rho, eta_rho) */
    const int32_t *mask_u;       /* (xi_u, eta_u) */
    const int32_t *mask_v;       /* (xi_v, eta_v) */
    const double *s_rho, *cs_r;  /* (N)   */
    const double *s_w, *cs_w;    /* (N+1) */
    double scl[ORC_MAXNGRID][2]; /* GRIDS(ng)%scl(i,1:2): map to grid i */
    double off[ORC_MAXNGRID][2]; /* GRIDS(ng)%off(i,1:2)               */
    /* HYDRODATA(ng)%<field>(:,:,:,tind) for tind = 1..3 */
    const double *zeta[3], *u[3], *v[3], *w[3], *aks[3];
    /* diagnostics fields (NULL unless used): salt, temp (xi_rho,eta_rho,N),
     * bustr (xi_u,eta_u), bvstr (xi_v,eta_v) */
    const double *salt[3], *temp[3], *bustr[3], *bvstr[3];
    /* GRIDS(ng)%lon_rho, lat_rho (xi_rho, eta_rho); NULL unless output is used */
    const double *lon_rho, *lat_rho;
    /* -DWETDRY: HYDRODATA(ng)%wetdry_mask_rho/_u/_v(:,:,tind); when set,
     * getInterp3D and getInterpStr take their masks from these
     * (hydrodynamic_module.f90:510-570); NULL: the static grid masks */
    const double *wd_rho[3], *wd_u[3], *wd_v[3];
    /* behaviour fields (Process_VA / Process_WA), (xi_rho,eta_rho,N+1):
     * HYDRODATA(ng)%Accelstd_t, Vortstd_t, Accelustd_w, Accelvstd_w */
    const double *turbaccel[3], *turbvort[3], *waveaccelu[3], *waveaccelv[3];
    /* GRIDS(ng)%angle (xi_rho, eta_rho) for LL2ij (NULL unless used) */
    const double *angle;
} orc_grid;

typedef struct {
    int ngrid;
    int idt;                     /* internal step (s), INTEGER in ROMSPath.h */
    int scheme;                  /* 1 = RK4 */
    int nsb;                     /* 0 neutral, 1 surface, 2 bottom */
    int vturb_on, hturb_on, open_ocean_boundary;
    double vertdist, serr, smth, sub, deltat, aksback;
    double constant_hturb[ORC_MAXNGRID];
    int spline_max_iter;         /* cap on smooth()'s secant loop (ref: none) */
    int salttemp_on, salttemp_mean, write_bottom;   /* SaltTempOn, SaltTempMean, WriteBottom */
    /* behave (behavior_module.f90:186-393): Behavior (0, 1 or 10),
     * Process_VA, Process_WA, va_flag; swimfast (m/s); initsize =
     * par(:,pSize); the fuchsparam namelist (ROMSPath.h:165-189) */
    int behavior, process_va, process_wa, va_flag;
    double swimfast, initsize;
    double vort_cr, vort_sat, b0pv, b1pv, b0wv, b1w, acc_cr, acc_sat, b0pa, b1pa, b0wa;
    /* Experiment variants of VTurb for attributing well-mixed-condition
     * results (0 / NaN: the reference's algorithm).  vt_variant 1 replaces
     * the smoothing-spline fit by the parabola K = c 4 xi (1 - xi),
     * xi = (z - tdepth) / (zeta - tdepth), with c the least-squares fit to
     * the column, and K' its exact derivative; vt_dy_end, when not NaN, is
     * the value of dy(1) and dy(np) (never set by the reference,
     * ver_turb_module.f90:131-136; pinned to serr otherwise). */
    int vt_variant;
    double vt_dy_end;
} orc_params;

typedef struct {
    int64_t n;
    double *x, *y, *z, *dob, *age, *status; /* par(:,pX/pY/pZ/pDOB/pAge/pStatus) */
    int32_t *gid;                            /* int(par(:,pGID)) */
    int8_t *isin;                            /* isIn(:) */
    double *wd, *zeta, *bath;                /* par(:,pWD/pZeta/pBath) */
    uint32_t *flags;
    const uint32_t *pid;                     /* persistent particle id (noise) */
    /* diagnostics (NULL unless used): P_Salt, P_Temp, mean_salt, mean_temp,
     * P_HOB, P_bustr, P_bvstr (ROMSPath.f90:130-131) */
    double *p_salt, *p_temp, *mean_salt, *mean_temp, *p_hob, *p_bustr, *p_bvstr;
    /* behave's outputs par(:,pAcc/pVort/pbehaveW/pSSF) (NULL unless used) */
    double *p_acc, *p_vort, *p_behavew, *p_ssf;
} orc_particles;

/* MT19937 state, restated from random_module.f90:109-198. */
typedef struct {
    uint32_t mt[624];
    int mti;
} orc_mt19937;

enum { ORC_NOISE_MT = 0, ORC_NOISE_PHILOX = 1, ORC_NOISE_HOOK = 2 };

typedef struct {
    int kind;
    orc_mt19937 *mt;             /* ORC_NOISE_MT: one global serial stream */
    uint64_t seed;               /* ORC_NOISE_PHILOX: key                  */
    uint64_t step;               /* ORC_NOISE_PHILOX: internal-step index  */
    const double *hook;          /* ORC_NOISE_HOOK: hook[pid*ndraw + d]    */
    int ndraw;                   /* draws per particle per step in hook    */
} orc_noise;

/* ---- primitives (exported for unit tests) ---- */
void     orc_mt_init(orc_mt19937 *s, uint32_t seed);
uint32_t orc_mt_int32(orc_mt19937 *s);
double   orc_mt_real3(orc_mt19937 *s);
void     orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
double   orc_philox_normal(uint64_t seed, uint32_t pid, uint64_t step, uint32_t draw);
double   orc_log_pos(double x);
double   orc_cos2pi(double u);
/* exp and log of any double from their series with exact argument
 * reductions (own restatement; the device uses the same operations) */
double   orc_exp(double x);
double   orc_log(double x);
/* the k-th uniform (k = 0..4) of behave's draws under Philox: counter
 * (pid, step, 0x40000000 + k/4), word k%4, (r + 0.5) / 2^32 */
double   orc_philox_uniform(uint64_t seed, uint32_t pid, uint64_t step, uint32_t k);

double orc_polintd(const double xa[3], const double ya[3], double x);
void   orc_linint(const double *xa, const double *ya, int n, double x, double *y, double *m);
double orc_getslevel(const orc_grid *g, double zeta, double depth, int k);
double orc_getwlevel(const orc_grid *g, double zeta, double depth, int k);
int    orc_inside(int nb, double *xb, double *yb, double xo, double yo);
void   orc_bounds(const orc_grid *g, double ipar, double jpar, int *nmask,
                  int *ingrid, int *obound);
double orc_getinterp2d(const orc_grid *g, int var, double ipar, double jpar,
                       int t, uint32_t *flags);
double orc_getinterp3d(const orc_grid *g, int var, double ipar, double jpar,
                       double zpar, int t, int ztype, double zeta,
                       double depth, uint32_t *flags);
/* smooth(): returns sfq; a is (np,4) column-major output; v is (np,7)
 * workspace; *iters receives the number of secant iterations. */
double orc_smooth(const double *x, const double *y, const double *dy, int np,
                  double s, double *v, double *a, int max_iter, int *iters);
double orc_ppvalu(const double *brk, const double *coef, int l, int k,
                  double x, int jderiv);

/* 2-D variable ids for orc_getinterp2d / 3-D ids for orc_getinterp3d */
enum { ORC_V_DEPTH = 0, ORC_V_PM, ORC_V_PN, ORC_V_ZETA, ORC_V_LON, ORC_V_LAT };
enum { ORC_V_U = 0, ORC_V_V, ORC_V_W, ORC_V_AKS, ORC_V_SALT, ORC_V_TEMP,
       ORC_V_TURBACCEL, ORC_V_TURBVORT, ORC_V_WAVEACCELU, ORC_V_WAVEACCELV };
/* getInterpStr variables (interpolation_module.f90:964-1174) */
enum { ORC_V_BUSTR = 0, ORC_V_BVSTR };
double orc_getinterp_str(const orc_grid *g, int var, double ipar, double jpar, int t, uint32_t *flags);

/* ---- the particle step (update_particles, ROMSPath.f90:608-1008) ---- */
int orc_update_particles(const orc_params *prm, const orc_grid *grids,
                         orc_particles *p, const double ex[3],
                         const double ix[3], int ets, int tb, int tc, int tf,
                         const orc_noise *noise, int nthreads);

/* Init-time ownership test of ini_ROMSPath (ROMSPath.f90:367-432): for
 * positions already in index space of each grid, first grid whose bounds()
 * says in-grid owns the particle; zbounds() fixes z.  ipos/jpos are
 * (ngrid, n) row-major: ipos[g*n + k].  With SaltTempOn the initial salt,
 * temp (and pWD/pZeta/pBath) are taken at ring slot tc (408-427). */
int orc_init_particles(const orc_params *prm, const orc_grid *grids,
                       orc_particles *p, const double *ipos,
                       const double *jpos, int tb, int tc);

/* dataOutput (ROMSPath.f90:1012-1024): pLon, pLat by getInterp2D("lon"/
 * "lat", pGID, pX, pY, 1) for every particle (gather indices clamped; no
 * flag is recorded, as the output step changes no particle state). */
void orc_output_lonlat(const orc_grid *grids, const orc_particles *p, double *lon, double *lat);

/* sin, cos (|x| < 2^19 pi/2) and asin from their series with exact
 * argument reductions (own restatement; the device runs the same ops) */
void   orc_sincos(double x, double *s, double *c);
double orc_asin(double x);

/* LL2ij (interpolation_module.f90:110-231) for particles at (inlon,
 * inlat) in grid g: bisection of the grid with inbox (232-268) and inside,
 * then the Cartesian (spherical = 0) or spherical (1) fractional index;
 * spherical is GRIDS(1)%spherical, as the reference reads it. */
void orc_ll2ij(const orc_grid *g, int spherical, const double *inlon, const double *inlat, int64_t n,
               double *ipar, double *jpar);

/* The nest maps of InitGrid (grid_module.f90:441-481): grefine from
 * refine(1..Ngrid-1), the first coincident lon/lat rho point of each grid
 * pair by the reference's search order, and scl/off of every pair; scl and
 * off are [ng][2][Ngrid] (GRIDS(ng)%scl(i,c) at [ng][c][i]). */
void orc_nest_maps(int ngrid, const orc_grid *grids, const double *refine, double *scl, double *off);

/* statistics of the last orc_update_particles call (secant iterations) */
void orc_last_stats(int64_t *spline_calls, int64_t *secant_iters);

#ifdef __cplusplus
}
#endif
#endif
