/*
 * romspath_gpu.h -- C ABI of the B200 ROMSPath particle step.
 *
 * Drop-in for the body of update_particles (ROMSPath.f90:608-1008) and the
 * frame hand-off of updateHydro (hydrodynamic_module.f90:112-760).  The
 * Fortran driver, its namelists (ROMSPath.h:59-345) and its NetCDF reader
 * stay as they are; the driver binds these entry points with ISO_C_BINDING
 * (one bind(C) interface per entry point, arguments by value or as arrays).
 *
 * Conventions
 *  - Every array argument is a host pointer in the reference's own layout:
 *    Fortran column-major, 1-based index semantics.  h(xi_rho,eta_rho),
 *    U(xi_u,eta_u,N), V(xi_v,eta_v,N), W/AKs(xi_rho,eta_rho,N+1),
 *    zeta(xi_rho,eta_rho) with xi_u = xi_rho-1, eta_u = eta_rho,
 *    xi_v = xi_rho, eta_v = eta_rho-1.  Arrays are borrowed for the call.
 *  - Slots are the reference's ring positions tind = 1..3 (t_b/t_c/t_f).
 *  - Grid ids are 1..Ngrid, as par(:,pGID).
 *  - Every call returns RP_OK (0) or a negative RP_ERR_* code; the message
 *    of the last error is available from rp_last_error().  No call exits or
 *    aborts the process.
 *  - One host thread drives a context.  rp_step() and rp_upload_frame*()
 *    are asynchronous (stream-ordered); rp_get_particles() and
 *    rp_synchronize() wait for the device.
 */
#ifndef ROMSPATH_GPU_H
#define ROMSPATH_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RP_MAXNGRID 5          /* MAXNgrid, ROMSPath.h:9 */

#define RP_OK 0
#define RP_ERR_ARG (-1)        /* bad argument, dimension, slot or grid id   */
#define RP_ERR_CUDA (-2)       /* CUDA runtime error (message has details)   */
#define RP_ERR_STATE (-3)      /* call made in the wrong order               */
#define RP_ERR_NOMEM (-4)      /* device or pinned allocation failed         */
#define RP_ERR_UNSUPPORTED (-5)/* option outside the implemented path        */
#define RP_ERR_NOEXT (-6)      /* no CUDA device / kernels not loadable      */

/* per-particle flag bits returned by rp_get_particles: each marks a particle
 * that met, in its steps, a case where the reference's result is undefined
 * and this library pins one (the bits below say which) */
#define RP_FLAG_OOB 0x01u      /* a gather index left its array (clamped)      */
#define RP_FLAG_NODE 0x02u     /* inverse-distance weight at an exact node      */
#define RP_FLAG_WBOT 0x04u     /* w-level bracket below level 1                 */
#define RP_FLAG_WTOP 0x08u     /* w-level bracket above level N+1               */
#define RP_FLAG_SPLINE 0x10u   /* smoothing-spline secant loop hit its cap      */

/* storage precision of the hydrodynamic fields on the device */
#define RP_FIELD_F64 0
#define RP_FIELD_F32 1
/* The mixed-precision form: u, v, w, AKs stored in FP16 with a power-of-two
 * scale per (slot, level), zeta in FP32; positions in FP32 with Kahan-
 * compensated accumulation; interpolation and RK4 in FP32; age, the
 * smoothing spline's factor rows and secant search and the random-
 * displacement sub-steps in FP64, the spline's substitution sweeps in
 * FP32, with its smoothing parameter extrapolated from the particle's
 * previous two steps.  Non-finite field values are stored as finite ones
 * (FP16: NaN as 0, +-Inf as +-65504; int16: clamped).  Not bit-exact; its error against RP_FIELD_F64 on the
 * same noise is measured by the tests. */
#define RP_FIELD_MIXED 2
/* The same form with u, v, w, AKs in int16 fixed point, scale = level
 * max / 32767 (15 bits for the largest values of a level, where FP16 keeps
 * 11; absolute rather than relative resolution below them). */
#define RP_FIELD_MIXED_I16 3

/* Diagnostics switches, rp_params.reserved[3] (namelist "other",
 * ROMSPath.h:325-330; computed at the end of update_particles' particle
 * loop, ROMSPath.f90:935-986).  Every form; the mixed forms hold the
 * diagnostics' fields in FP32. */
#define RP_DIAG_SALTTEMP 1       /* SaltTempOn: P_Salt, P_Temp               */
#define RP_DIAG_SALTTEMP_MEAN 2  /* SaltTempMean: their running sums         */
#define RP_DIAG_BOTTOM 4         /* WriteBottom: P_HOB, P_bustr, P_bvstr     */

/* Run parameters: the namelist values the hot path reads (ROMSPath.h:77-80
 * timeparam, 140-148 turbparam, 152-154 advectparam, 161-180 behavparam,
 * 304-319 other) plus device options. */
typedef struct rp_params {
    int32_t numpar;                      /* particle capacity (numparticles)  */
    int32_t idt;                         /* internal step (s)                 */
    int32_t dt;                          /* external step (s)                 */
    int32_t scheme;                      /* 1 = RK4, else no advection        */
    int32_t nsb;                         /* 0 neutral, 1 surface, 2 bottom    */
    int32_t vturb_on;                    /* VTurbOn                           */
    int32_t hturb_on;                    /* HTurbOn                           */
    int32_t open_ocean_boundary;         /* OpenOceanBoundary                 */
    int32_t behavior;                    /* Behavior: 0 passive, 1 swim, 10 Fuchs,
                                            11 none (VA output); rp_set_behavior
                                            for the others' parameters       */
    int32_t stokes;                      /* add ustokes/vstokes on upload     */
    int32_t field_dtype;                 /* RP_FIELD_F64 / _F32 / _MIXED      */
    int32_t spline_max_iter;             /* cap of smooth()'s secant loop (0: 100) */
    double vertdist;
    double serr, smth, sub, deltat, aksback;
    double constant_hturb[RP_MAXNGRID];  /* ConstantHTurb(ng), m^2/s          */
    uint64_t seed;                       /* Philox key of the turbulence noise */
    int32_t device;                      /* CUDA device ordinal               */
    int32_t reserved[7];                 /* [0]: kernel form, 0 fused (default),
                                            1 split, 2 shared-memory split,
                                            3 fused without load-ahead, 4/5
                                            fused in 64/256-thread blocks
                                            (mixed forms; rp_set_kernel_form);
                                            [1]: re-sort the particle
                                            state by grid and cell every that
                                            many internal steps (0: never;
                                            results are unchanged, gathers
                                            coalesce); [2]: cap on resident
                                            blocks per SM of the step kernels
                                            (0: the occupancy limit; sets the
                                            particles per thread); [3]:
                                            diagnostics, RP_DIAG_* bits;
                                            [4]: 1 = WETDRY (the -DWETDRY
                                            build: per-frame wet/dry masks
                                            in getInterp3D and
                                            getInterpStr; every form);
                                            others 0 */
} rp_params;

/* One grid (GRIDS(ng), grid_module.f90:14-35).  Pointers are borrowed for
 * the duration of rp_create(). */
typedef struct rp_grid {
    int32_t xi_rho, eta_rho;             /* rho-point dimensions              */
    int32_t n_rho;                       /* s_rho (N), 2..510; s_w = N+1      */
    int32_t vtransform;                  /* 1, 2 or 3                         */
    double hc;
    const double *h, *pm, *pn;           /* (xi_rho, eta_rho)                 */
    const int32_t *mask_rho;             /* (xi_rho, eta_rho)                 */
    const int32_t *mask_u;               /* (xi_u, eta_u)                     */
    const int32_t *mask_v;               /* (xi_v, eta_v)                     */
    const double *s_rho, *cs_r;          /* (N)                               */
    const double *s_w, *cs_w;            /* (N+1)                             */
    const double *scl, *off;             /* scl(Ngrid,2), off(Ngrid,2), Fortran order;
                                            NULL for a single grid           */
} rp_grid;

typedef struct rp_ctx rp_ctx;

/* Create a context on params->device: uploads the static grids and sizes
 * the frame ring and particle state.  Replaces the device-side part of
 * ini_ROMSPath (ROMSPath.f90:182-461; GRIDS from InitGrid,
 * grid_module.f90:41-499). */
int rp_create(const rp_params *params, int32_t ngrid, const rp_grid *grids, rp_ctx **out);

/* Hand one frame of grid `ng` (1..Ngrid) to ring slot `slot` (1..3): the
 * output of updateHydro(FIRST, tstep, tind) (hydrodynamic_module.f90:112-760)
 * for tind = slot.  zeta(xi_rho,eta_rho), u(xi_u,eta_u,N), v(xi_v,eta_v,N),
 * w and aks (xi_rho,eta_rho,N+1); su/sv are ustokes/vstokes (may be NULL;
 * added to u/v in FP64 when params->stokes, hydrodynamic_module.f90:606-660).
 * The copy runs asynchronously into a spare device slot; the arrays may be
 * reused as soon as the call returns. */
int rp_upload_frame(rp_ctx *ctx, int32_t ng, int32_t slot, const double *zeta, const double *u,
                    const double *v, const double *w, const double *aks, const double *su,
                    const double *sv);
/* Same for single-precision source arrays. */
int rp_upload_frame_f32(rp_ctx *ctx, int32_t ng, int32_t slot, const float *zeta, const float *u,
                        const float *v, const float *w, const float *aks, const float *su,
                        const float *sv);

/* rp_upload_frame with the fields of the diagnostics: salt and temp
 * (xi_rho,eta_rho,N) for RP_DIAG_SALTTEMP, bustr (xi_u,eta_u) and bvstr
 * (xi_v,eta_v) for RP_DIAG_BOTTOM (hydrodynamic_module.f90:262-450; the
 * caller adds TempOffset, as updateHydro does).  With a diagnostic on, its
 * fields are required on every upload and rp_upload_frame refuses. */
int rp_upload_frame_ext(rp_ctx *ctx, int32_t ng, int32_t slot, const double *zeta, const double *u,
                        const double *v, const double *w, const double *aks, const double *su,
                        const double *sv, const double *salt, const double *temp, const double *bustr,
                        const double *bvstr);
int rp_upload_frame_ext_f32(rp_ctx *ctx, int32_t ng, int32_t slot, const float *zeta, const float *u,
                            const float *v, const float *w, const float *aks, const float *su,
                            const float *sv, const float *salt, const float *temp, const float *bustr,
                            const float *bvstr);

/* Every field of a frame in one descriptor: the pointers are const
 * double * (f32 = 0) or const float * (f32 = 1); zeta..aks required,
 * su/sv with params->stokes, salt..bvstr with the diagnostics, and the
 * WETDRY masks HYDRODATA(ng)%wetdry_mask_rho/_u/_v(:,:,tind) (0/1 doubles,
 * (xi_rho,eta_rho), (xi_u,eta_u), (xi_v,eta_v); hydrodynamic_module.f90:
 * 510-570) with reserved[4] = 1.  NULL where unused. */
typedef struct rp_frame {
    int32_t f32;
    const void *zeta, *u, *v, *w, *aks;
    const void *su, *sv;
    const void *salt, *temp, *bustr, *bvstr;
    const double *wetdry_rho, *wetdry_u, *wetdry_v;
    /* behave's fields, (xi_rho,eta_rho,N+1): Accelstd_t and Vortstd_t with
     * Process_VA, Accelustd_w and Accelvstd_w with Process_WA
     * (hydrodynamic_module.f90:662-760) */
    const void *turbaccel, *turbvort, *waveaccelu, *waveaccelv;
} rp_frame;
int rp_upload_frame_desc(rp_ctx *ctx, int32_t ng, int32_t slot, const rp_frame *frame);

/* Set the particle state: the par(:,pX/pY/pZ/pDOB/pAge/pStatus/pGID)
 * columns and isIn(:) of ROMSPath.f90:104-129 for particles 1..n. */
int rp_set_particles(rp_ctx *ctx, int64_t n, const double *x, const double *y, const double *z,
                     const double *dob, const double *age, const double *status, const double *gid,
                     const int32_t *isin);

/* Initial ownership: the grid loop of ini_ROMSPath (ROMSPath.f90:367-432)
 * with bounds() and zbounds() on the device.  ipos/jpos are (n, Ngrid)
 * Fortran order (particle positions in each grid's index space, the output
 * of LL2ij); z and dob are par(:,pZ) and par(:,pDOB). */
int rp_locate_particles(rp_ctx *ctx, int64_t n, const double *ipos, const double *jpos,
                        const double *z, const double *dob, int32_t t_b);

/* GRIDS(ng)%angle (xi_rho,eta_rho; radians, may be NULL for a Cartesian
 * grid) and GRIDS(ng)%spherical (0 or 1) for rp_locate_lonlat
 * (grid_module.f90:225-300). */
int rp_set_grid_angle(rp_ctx *ctx, int32_t ng, const double *angle, int32_t spherical);

/* rp_locate_particles from the particles' lon/lat (the parfile columns,
 * ROMSPath.f90:319-356): LL2ij (interpolation_module.f90:110-268: a
 * bisection of each grid with the point-in-polygon test inbox, then the
 * Cartesian or spherical fractional index, GRIDS(1)%spherical deciding for
 * every grid) of every particle in every grid on the device, then the
 * ownership loop.  rp_set_grid_lonlat and rp_set_grid_angle first.
 * ipos_out/jpos_out (may be NULL) receive the (n, Ngrid) Fortran-order
 * indices LL2ij gave. */
int rp_locate_lonlat(rp_ctx *ctx, int64_t n, const double *lon, const double *lat, const double *z,
                     const double *dob, int32_t t_b, double *ipos_out, double *jpos_out);

/* InitGrid's nest maps (grid_module.f90:437-481), host only: grefine(a,b) =
 * refine(|a-b|)^|a-b|, and for every grid pair the first coincident lon/lat
 * rho point in the reference's search order (found by hashing, O(points)
 * instead of the reference's O(points^2)); scl and off receive, per grid
 * ng, GRIDS(ng)%scl(Ngrid,2) and off(Ngrid,2) in Fortran order at
 * scl + ng*2*Ngrid -- what rp_grid.scl/off take.  Without a coincident
 * point the indices are those past the search loops' ends, as in the
 * reference. */
int rp_nest_maps(int32_t ngrid, const int32_t *xi_rho, const int32_t *eta_rho, const double *const *lon_rho,
                 const double *const *lat_rho, const double *refine, double *scl, double *off);

/* One internal step over all particles: update_particles
 * (ROMSPath.f90:608-1008) with ex(3), ix(3), ets and the ring slots
 * t_b/t_c/t_f from run_External_Timestep / run_Internal_Timestep
 * (ROMSPath.f90:465-546). */
int rp_step(rp_ctx *ctx, const double ex[3], const double ix[3], int32_t ets, int32_t t_b,
            int32_t t_c, int32_t t_f);

/* `nsteps` internal steps in one call (typically the 12 of one external
 * step, run_Internal_Timestep's loop, ROMSPath.f90:517-530): ex, ix are
 * [nsteps][3], ets and the slots [nsteps].  The steps' launches are
 * captured into a CUDA graph and launched as one; the graph of the previous
 * call is updated in place when it has the same shape.  Same results as
 * nsteps calls of rp_step. */
int rp_step_n(rp_ctx *ctx, int32_t nsteps, const double *ex, const double *ix, const int32_t *ets,
              const int32_t *t_b, const int32_t *t_c, const int32_t *t_f);

/* Read back par(:,pX/pY/pZ/pAge/pStatus/pGID), isIn, par(:,pWD/pZeta/pBath)
 * and the per-particle flag bits for particles 1..n.  Any pointer may be
 * NULL.  Waits for queued work. */
int rp_get_particles(rp_ctx *ctx, int64_t n, double *x, double *y, double *z, double *age,
                     double *status, double *gid, int32_t *isin, double *wd, double *zeta,
                     double *bath, uint32_t *flags);

/* behave (behavior_module.f90:186-393): the behavparam / fuchsparam
 * namelists (ROMSPath.h:150-189) and par(:,pSize) = initsize (199, 342).
 * behavior must equal rp_params.behavior.  Process_VA / Process_WA add
 * their fields to every frame (rp_upload_frame_desc) and draw, per
 * particle-step, 4 Laplace, 2 normal and 1 uniform deviates; Behavior 1
 * adds swimfast*idt, Behavior 10 the Fuchs swim/sink velocity*idt to the
 * vertical displacement.  Call before the first frame upload and before
 * rp_set_noise_hook (the hook then holds 2 + idt/deltat + 7 draws per
 * particle-step: behave's two normals, then its five uniforms in (0,1)).
 * Every form; the mixed forms hold behave's fields in FP32. */
typedef struct rp_behavior {
    int32_t behavior, process_va, process_wa, va_flag;
    double swimfast;                     /* m/s (Behavior 1)                  */
    double initsize;                     /* larval size (um)                  */
    double vort_cr, vort_sat, b0pv, b1pv, b0wv, b1w;
    double acc_cr, acc_sat, b0pa, b1pa, b0wa;
} rp_behavior;
int rp_set_behavior(rp_ctx *ctx, const rp_behavior *b);

/* Read back par(:,pAcc/pVort/pbehaveW/pSSF) (ROMSPath.f90:800-804) for
 * particles 1..n; zeros without Process_VA / _WA.  Any pointer may be NULL.
 * Waits for queued work. */
int rp_get_behavior(rp_ctx *ctx, int64_t n, double *acc, double *vort, double *behavew, double *ssf);

/* Read back the diagnostics for particles 1..n: P_Salt, P_Temp,
 * mean_salt, mean_temp (the running sums: the writer divides them by its
 * count mI, ROMSPath.f90:2010-2014), P_HOB, P_bustr, P_bvstr.  Any pointer
 * may be NULL; asking for a diagnostic that is off is RP_ERR_STATE.  Waits
 * for queued work.  rp_set_particles sets them as the particle read loop
 * does (P_HOB 9999, the others 0); rp_locate_particles also computes the
 * initial salinity and temperature from slot t_b % 3 + 1 (t_c), with
 * par(:,pWD/pZeta/pBath), as ini_ROMSPath does (ROMSPath.f90:408-427). */
int rp_get_diagnostics(rp_ctx *ctx, int64_t n, double *salt, double *temp, double *mean_salt,
                       double *mean_temp, double *hob, double *bustr, double *bvstr);

/* The writer's resets after an output record (ROMSPath.f90:2030-2035,
 * 2064): mean_salt, mean_temp to 0 and P_HOB to 9999.  Stream-ordered. */
int rp_reset_diagnostics(rp_ctx *ctx);

/* GRIDS(ng)%lon_rho, lat_rho (xi_rho,eta_rho) of grid ng, for the output
 * records (grid_module.f90:209-300). */
int rp_set_grid_lonlat(rp_ctx *ctx, int32_t ng, const double *lon_rho, const double *lat_rho);

/* One output record: dataOutput (ROMSPath.f90:1012-1024) and the columns
 * writeNetCDF puts (1924-2070), computed on the device for particles 1..n
 * in the caller's order: lon, lat (getInterp2D "lon"/"lat", plain bilinear
 * at pGID, pX, pY; rp_set_grid_lonlat first), zp = par(:,pZ), age, status,
 * GID; salt and temp (mean_salt/mI, mean_temp/mI under SaltTempMean, else
 * P_Salt/P_Temp); HOB, bustr, bvstr.  Then the writer's resets: the sums to
 * 0 (SaltTempMean) and P_HOB to 9999 (WriteBottom), for every particle,
 * whichever columns were asked for.  mI is the driver's step count since
 * the last record (ROMSPath.f90:422, 533, 2035).  Any pointer may be NULL.
 * Waits for queued work. */
int rp_output_record(rp_ctx *ctx, int64_t n, int32_t mI, double *lon, double *lat, double *zp,
                     double *age, double *status, double *gid, double *salt, double *temp,
                     double *hob, double *bustr, double *bvstr);

/* rp_output_record without waiting: the record is packed in stream order
 * (after the steps queued so far, with the writer's resets) and its
 * columns are copied into the caller's arrays, which must be page-locked,
 * on a stream of their own while the steps queued next run.  The arrays
 * may be read (or reused) only after rp_output_wait (or rp_synchronize).
 * A later record waits for this one's copies before it is packed. */
int rp_output_record_async(rp_ctx *ctx, int64_t n, int32_t mI, double *lon, double *lat, double *zp,
                           double *age, double *status, double *gid, double *salt, double *temp,
                           double *hob, double *bustr, double *bvstr);

/* Wait for the copies of the last rp_output_record_async. */
int rp_output_wait(rp_ctx *ctx);

/* First particle id of this context (default 0).  Particle k of the next
 * rp_set_particles / rp_locate_particles call gets id base + k; the id keys
 * its Philox noise, so a run split over several contexts (one per GPU) with
 * disjoint id ranges draws the same noise as one context holding all
 * particles.  The noise hook is indexed by id - base. */
int rp_set_id_base(rp_ctx *ctx, uint32_t base);

/* Index of the next internal step in the Philox counter (default 0; each
 * rp_step increments it). */
int rp_set_step_index(rp_ctx *ctx, uint64_t step_index);

/* Test hook: replace the Philox normals by caller-supplied N(0,1) values,
 * laid out [step][particle][draw] with draw = 0,1 for HTurb (devX, devY)
 * and 2..1+idt/deltat for the VTurb sub-steps; `nsteps` steps are held.
 * NULL removes the hook. */
int rp_set_noise_hook(rp_ctx *ctx, const double *noise, int64_t nsteps);

/* Wait for all queued work of the context. */
int rp_synchronize(rp_ctx *ctx);

/* Copy the last error message (NUL-terminated, truncated to len). */
int rp_last_error(rp_ctx *ctx, char *buf, int32_t len);

/* Release the context and its device memory. */
int rp_destroy(rp_ctx *ctx);

/* Device-resident state, for callers that keep particles in HBM between
 * calls (pointers stay valid until rp_destroy).  With re-sorting on
 * (rp_params.reserved[1]) the columns are in the library's order: pid[i]
 * minus the id base of the particle set is particle i's index.  In the mixed form the
 * positions live in compensated FP32 columns: rp_device_state_get first
 * writes x, y, z from them (and waits), and the mixed step does not read
 * x, y, z back. */
typedef struct rp_device_state {
    int64_t n;
    double *x, *y, *z, *age, *dob, *status, *wd, *zeta, *bath;
    int32_t *gid;
    int8_t *isin;
    uint32_t *pid, *flags;
    void *stream;                        /* cudaStream_t of the compute stream */
} rp_device_state;
int rp_device_state_get(rp_ctx *ctx, rp_device_state *out);

/* Largest particle count rp_step_noalloc accepts: its scratch is a fixed
 * device buffer of one double per particle (8 MiB). */
#define RP_NOALLOC_MAX_PARTICLES 1048576

/* One internal step exactly like rp_step (same results, bit for bit), on
 * particle columns that live in the caller's own device memory
 * (state->x ... state->flags, state->n particles), and without allocating
 * any device memory.  No counterpart in the reference.
 *
 * For callers that cannot allocate at step time: a Fortran driver that keeps
 * its particle arrays on the device itself (OpenACC / CUDA Fortran data
 * regions) within its own memory budget, a host framework whose allocator
 * owns the device's memory, or a time loop that must not call cudaMalloc
 * because it synchronises the device and stalls the asynchronous frame
 * uploads.  The one scratch array the step needs (the VTurb displacement of
 * each particle) is a fixed 8 MiB device buffer that exists on every device
 * that loads the library until the process exits.
 *  - state->n must be <= RP_NOALLOC_MAX_PARTICLES and int(s_w*sub) <= 128
 *    (RP_ERR_ARG / RP_ERR_UNSUPPORTED otherwise, with a message).
 *  - state->stream is the caller's stream that orders its own reads and
 *    writes of the columns (NULL: the legacy default stream).  The step
 *    runs on the context's compute stream after the work queued on
 *    state->stream so far, and work queued on state->stream after the call
 *    runs after the step; with state->stream equal to the compute stream
 *    (as rp_device_state_get returns it) nothing extra is ordered.
 *  - The first call on a device looks up the buffer's device address; make
 *    that first call before any stream capture.  A process that resets the
 *    device (cudaDeviceReset) between calls is not supported: the address
 *    is kept for the life of the process.
 *  - Calls share the buffer: calls that overlap on the GPU (other streams or
 *    threads) race and must be serialised by the caller.  Its contents are
 *    never read before the same call writes them, so nothing is cleared.
 *  - The noise hook is not used by this entry point (RP_ERR_STATE if set).
 *  - FP64 and FP32 field storage only (RP_ERR_UNSUPPORTED for RP_FIELD_MIXED).
 * Launches on the context's compute stream, after pending frame uploads. */
int rp_step_noalloc(rp_ctx *ctx, const rp_device_state *state, const double ex[3], const double ix[3],
                    int32_t ets, int32_t t_b, int32_t t_c, int32_t t_f);

/* ------------------------------------------------------------------------
 * Adjoint pair.  No counterpart in the reference (ROMSPath has no
 * derivative code): gradients of a loss of the final particle positions
 * with respect to each particle's initial position and to a multiplier
 * kappa of the vertical diffusivity AKs, for release attribution.
 *
 * The differentiated model is the FP64 step of update_particles
 * (ROMSPath.f90:662-905) with kappa scaling the AKs data, the smoothing
 * spline on uniform breaks, and frozen Philox noise.  rp_forward searches
 * each fit's smoothing parameter as smooth() does (pppack.f90:5108-5317)
 * and records it; rp_backward, rp_tangent and rp_adj_replay reuse the
 * recorded values, so the derivatives are those of the trajectory's own
 * piece (level brackets, reflections, land rejection and hand-off are taken
 * on values as well).  Frames come from a store that holds the whole time
 * window, since the backward sweep runs through it in reverse.
 * ---------------------------------------------------------------------- */
typedef struct rp_adj_step {
    double ex[3];                        /* frame times, as rp_step          */
    double ix[3];                        /* internal times, as rp_step       */
    int32_t ets;
    int32_t frame_b, frame_c, frame_f;   /* frames (1..nframes) in time slots b, c, f */
    uint64_t step_index;                 /* Philox step counter               */
} rp_adj_step;

/* Allocate the frame store for `nframes` frames of every grid (FP64). */
int rp_adj_frames(rp_ctx *ctx, int32_t nframes);
/* Frame number `frame` of grid `ng` into the store (arrays as
 * rp_upload_frame; Stokes added when params->stokes). */
int rp_adj_set_frame(rp_ctx *ctx, int32_t ng, int32_t frame, const double *zeta, const double *u,
                     const double *v, const double *w, const double *aks, const double *su,
                     const double *sv);
/* Run `nsteps` steps of the model from the current particle state
 * (rp_set_particles / rp_locate_particles), keeping the state every
 * `checkpoint_every` steps and the smoothing parameter of every fit.  The
 * final state is the context's particle state (rp_get_particles). */
int rp_forward(rp_ctx *ctx, int32_t nsteps, const rp_adj_step *steps, double kappa, int32_t checkpoint_every);
/* Given dL/d(final x, y, z) per particle, the gradients with respect to the
 * initial x, y, z (per particle) and to kappa (summed): reverse sweep over
 * the checkpoint segments, each segment's step-start states recomputed from
 * its checkpoint, each step's Jacobian applied transposed. */
int rp_backward(rp_ctx *ctx, const double *dL_dx, const double *dL_dy, const double *dL_dz, double *dL_dx0,
                double *dL_dy0, double *dL_dz0, double *dL_dkappa);
/* Tangent-linear reference: d(final x, y, z)/d(x0, y0, z0, kappa) per
 * particle by forward propagation, jac[n][3][4] (row x, y, z). */
int rp_tangent(rp_ctx *ctx, double kappa, double *jac);
/* The recorded run from other initial x, y, z (NULL: unchanged) and kappa,
 * with the recorded smoothing parameters: final x, y, z (for finite
 * differences). */
int rp_adj_replay(rp_ctx *ctx, const double *x0, const double *y0, const double *z0, double kappa, double *xf,
                  double *yf, double *zf);

/* Change the launch settings of rp_params.reserved[1] (re-sort interval,
 * 0: never) and [2] (resident blocks per SM, 0: occupancy limit) between
 * steps; results do not depend on them (an autotuner times real steps of
 * the run under each setting).  No counterpart in the reference. */
int rp_set_launch(rp_ctx *ctx, int32_t resort, int32_t blocks_per_sm);

/* Change the kernel form of rp_params.reserved[0] between steps: 0 fused
 * (one kernel per step, the fit's workspace in local memory), 1 split (a
 * VTurb kernel writing each particle's displacement, then the advection
 * kernel), and for the mixed forms 2, the split form with the VTurb
 * kernel's spline workspace in shared memory, 3, the fused kernel whose
 * back substitution does not load u ahead, and 4 and 5, the fused kernel
 * in blocks of 64 and 256 threads instead of 128 (the exact forms run 2-5
 * fused).  Results do not change beyond rounding (the exact forms:
 * not at all); which form is fastest depends on the grid and the particle
 * count, so an autotuner times them on the run.  No counterpart in the
 * reference. */
int rp_set_kernel_form(rp_ctx *ctx, int32_t form);

/* Timing of the last rp_step launch sequence on the compute stream, in ms
 * (CUDA events), and the number of kernels it launched. */
int rp_last_step_stats(rp_ctx *ctx, float *ms, int32_t *kernels);

/* Counting of VTurb's smoothing-spline fits (smooth, ver_turb_module.f90:182;
 * pppack.f90:5108-5317) and of the chol1d passes they make (pppack.f90:1428;
 * one per evaluation of SF in the secant search on p, plus the final u):
 * on = 1 zeroes the counts and counts the steps launched from then on,
 * on = 0 stops.  Counting adds one pair of atomic adds per warp and step;
 * it changes no result.  Every form; not in rp_forward/rp_backward. */
int rp_count_spline_passes(rp_ctx *ctx, int32_t on);

/* The counts since counting was last started (synchronises the compute
 * stream).  RP_ERR_STATE if it was never started. */
int rp_spline_pass_counts(rp_ctx *ctx, int64_t *fits, int64_t *passes);

/* Total number of kernels this context has launched since creation. */
int rp_kernel_launches(rp_ctx *ctx, int64_t *count);

/* Library version string. */
const char *rp_version(void);

#ifdef __cplusplus
}
#endif
#endif
