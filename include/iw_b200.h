/*
 * iw_b200.h -- C ABI of the B200 time-step library for the stratified
 * Boussinesq solver "Dubwise" (Fourier x,y / Legendre multidomain penalty z).
 *
 * Two groups of entry points:
 *
 *  1. The handle API (iw_*): a Fortran driver binds these with
 *     ISO_C_BINDING (every argument is a plain pointer or a value, every
 *     function returns an int status, 0 = ok).  Fields live on the device
 *     across steps; the host uploads the state once and downloads it for
 *     output or restart.
 *
 *  2. Drop-in replacements for the reference subroutines, with the
 *     reference's names, argument lists (all by reference, Fortran style,
 *     trailing underscore) and in-place semantics.  They act on the handle
 *     made current by iw_bind().  Routines that the reference calls on
 *     COMMON-block state (convec_, calcuvwt_) act on the bound handle's
 *     device state; routines that take an array argument (horfft_, dpdz_,
 *     interface_avg3d_, filter_3dlegenfourier_, ...) take host arrays and
 *     copy them in and out, as the reference's diagnostics need.
 *
 * Array layout (identical to the reference COMMON blocks): a field is
 * (nxpp, ny, nz) doubles, x fastest, with nxpp = nx+2.  In spectral space the
 * x index holds interleaved (Re, Im) pairs for kx = 0..nx/2, y holds FFT-
 * ordered ky, and z holds the physical GLL points of nsubd subdomains of nzloc
 * points each (interface points duplicated).  A column is the nz values of one
 * (kx, ky) mode.
 *
 * Threading: one host thread per handle; work is ordered on the handle's
 * CUDA stream.  Errors are reported by the return code and iw_last_error().
 */
#ifndef IW_B200_H
#define IW_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define IW_MAX_SUBD 64
#define IW_MAX_NZLOC 64

/* status codes */
#define IW_OK 0
#define IW_ERR_CONFIG 1    /* invalid dims / radices / subdomain table    */
#define IW_ERR_CUDA 2      /* a CUDA runtime call failed                  */
#define IW_ERR_NONFINITE 3 /* NaN/Inf detected in the state               */
#define IW_ERR_PIVOT 4     /* exactly zero pivot in a band factorisation  */
#define IW_ERR_STATE 5     /* call out of order (no handle bound, ...)    */
#define IW_ERR_NOMEM 6     /* device allocation failed                    */
#define IW_ERR_TIMEOUT 7   /* a bounded device wait gave up               */
#define IW_ERR_IO 8        /* a file could not be opened, read or written */

/* iw_read_restart modes */
#define IW_RESTART_EXACT 0     /* continue exactly where the writer stopped */
#define IW_RESTART_REFERENCE 1 /* main.f istart = 1 semantics               */

/* boundary-condition variants of calcuvwt (reference files in brackets) */
#define IW_BC_FREESLIP 0 /* calcuvwt.f / calcuvwt_freeslip.f: u,v Neumann at both ends */
#define IW_BC_NOSLIP 1   /* calcuvwt_noslip.f: u,v Dirichlet bottom, Neumann top      */

/* virtual paddle in rhsfm (solver.f:942-960), iw_params.forcing */
#define IW_PADDLE_OFF 0
#define IW_PADDLE_ALL_LEVELS 1  /* every z level, as the loop of solver.f:848 is written */
#define IW_PADDLE_ABOVE_BOTTOM 2 /* z levels 2..nz: the bottom point is left out, as the */
                                 /* comment at solver.f:848-849 says and as the reference's */
                                 /* recorded 400-step run (its log `output`, uveltest.dat */
                                 /* rows 641-1040) shows to 1e-10                          */

/* storage precision of the bulk fields */
#define IW_PREC_FP64 0  /* everything FP64 (parity path)                         */
#define IW_PREC_MIXED 1 /* FP32 fields/FFTs/products/filters, FP64 solves        */

/* vertical solves: AUTO = banded LU (the reference's SGBTRF/SGBTRS arithmetic)
 * for the pressure, subdomain block inverses + interface system for the
 * viscous and diffusive systems (FP32 inverses + one FP64 residual sweep in
 * the mixed path); LU = the reference's banded LU for every system. */
#define IW_SOLVE_AUTO 0
#define IW_SOLVE_LU 1

/* dim.h PARAMETERs, made runtime values (dim.h:12-28). */
typedef struct iw_dims {
  int32_t nx;    /* points in x (even; radices 2,3,5)            */
  int32_t ny;    /* points in y (1 => 2-D run, ndims=2)          */
  int32_t nzloc; /* GLL points per subdomain                     */
  int32_t nsubd; /* subdomains in z; nz = nzloc*nsubd            */
} iw_dims;

/* input.dat namelists &inputs &params &mflags (main.f:185-194) plus the
 * subd.dat table (setup.f:316-325) and the switches that the reference
 * hard-codes in source. */
typedef struct iw_params {
  /* &inputs */
  double dt;          /* dtin                                        */
  /* &params */
  double xlen, ylen, zlen;
  double brunt;       /* buoyancy frequency N                        */
  double xnu, xkappa; /* viscosity, diffusivity                      */
  double grav, rho0;
  double umax;        /* forcing velocity scale                      */
  double xacrit;      /* paddle forcing amplitude (0 = off)          */
  double xbcrit, zcen;/* mean-u damping window fzgaus                */
  double fwave;       /* forcing duration in wave periods            */
  /* &mflags */
  double amp, p, pf;  /* filter amplitude, Legendre/Fourier orders   */
  double fackc;
  double facdir, facneumn, facrobin;
  int32_t ispecfilternl, ispecfilterexp, nspecfilterexp, navgintrfc;
  /* switches hard-coded in the reference */
  int32_t bc_variant;    /* IW_BC_*                                  */
  int32_t meanu_damping; /* (1,1)-mode u *= 1-fzgaus (calcuvwt.f:343) */
  int32_t forcing;       /* IW_PADDLE_* (solver.f:942-960)           */
  int32_t precision;     /* IW_PREC_*                                */
  int32_t solver;        /* IW_SOLVE_AUTO or IW_SOLVE_LU             */
  int32_t imaxcalc;      /* 1: adaptive dt from the CFL numbers of   */
                         /* each step's start (main.f:47,657;        */
                         /* various.f:892-982); 0: dt fixed          */
  /* subd.dat */
  double z0[IW_MAX_SUBD];
  double zh[IW_MAX_SUBD];
} iw_params;

/* multistep coefficients (COMMON /ab/ /bdf/, comtimeadvance.h) */
typedef struct iw_coefs {
  double fac1, fac2, fac3;       /* SS extrapolation of the NL term */
  double bdf1, bdf2, bdf3, bdfv; /* BDF of the time derivative      */
  double dt;
} iw_coefs;

/* per-step diagnostics (maxcalc various.f:665-987, energycalc_postp
 * postp.f:415-732) */
typedef struct iw_diag_out {
  double ke;       /* 0.5 * sum_{k>=2} (u^2+v^2+w^2) over physical points */
  double eps;      /* xnu * sum_{k>=2} |grad u|^2                           */
  double umin, umax, vmin, vmax, wmin, wmax, tmin, tmax;
  double cflx, cfly, cflz;
  double wrms_bottom; /* rms of w over z < 0.2 zlen (noise growth)      */
  double t;
  double dt;          /* current step (changes only with imaxcalc = 1)  */
  int32_t istep;
  int32_t interface_avg_count[4];
} iw_diag_out;

typedef struct iw_handle iw_handle;

/* ---------------------------------------------------------------------- */
/* Handle API                                                               */
/* ---------------------------------------------------------------------- */

/* Replaces main.f:210-218 (fftfax/cftfax), setup.f:6-267 (setup) and the
 * allocation of every COMMON block; validates dims and the subdomain table.
 * device < 0 selects the current device. */
int iw_init(const iw_dims *dims, const iw_params *prm, int device,
            iw_handle **out);
int iw_destroy(iw_handle *h);
const char *iw_last_error(void);
/* Not in the reference.  The IW_ERR_* code of the last failure recorded on
 * this thread.  The reference-named routines that return nothing record
 * theirs here: penalty_main_ and bandlu_solve_ start from 0 and record
 * IW_ERR_PIVOT when SGBTF2 meets a zero pivot (its INFO, which the reference
 * ignores; the solution then holds Inf or NaN as the reference's would). */
int iw_last_status(void);

/* Upload / download the complete multistep state in the reference layout.
 * Each pointer addresses 4 fields (u,v,w,temp) back to back, i.e.
 * 4*nxpp*ny*nz doubles; NULL skips that level.  Levels: n, n-1, n-2 for the
 * prognostic fields (comflow.h) and n-1, n-2 for the NL terms (commatrix.h). */
int iw_upload_state(iw_handle *h, const double *uvwt, const double *uvwt_n,
                    const double *uvwt_nm, const double *s_n,
                    const double *s_nm, double t, int istep_done);
int iw_download_state(iw_handle *h, double *uvwt, double *uvwt_n,
                      double *uvwt_nm, double *s_n, double *s_nm);

/* Replaces output.f:2-117 (subroutine output, the restart dump of
 * main.f:974,988-989): writes the 49 records of output.f in its order and
 * sizes, as ifort unformatted sequential (4-byte little-endian byte counts
 * around each record; REAL*8 and INTEGER*4 items), so that restart.f reads
 * the file.  Records 30-49 hold the state levels n, n-1, n-2 and the NL terms
 * at n-1, n-2; the setup tables that the reference recomputes after a read
 * hold this library's tables or 0.  One more record follows, which restart.f
 * does not read: the step counter, the adaptive-step and restart state and
 * the multistep coefficients.  Records over 2147483639 bytes are refused. */
int iw_write_restart(iw_handle *h, const char *path);
/* Replaces restart.f:2-126 and main.f:555-632 (istart = 1 or 2).  Checks every
 * record's framing and size against the handle's dims before it changes
 * anything (the reference only warns on a dims mismatch: IW_ERR_CONFIG here).
 * mode IW_RESTART_REFERENCE: the reference's semantics -- t from the file,
 * the step counter from 0, and the first step's coefficients for a step dt
 * after two of cdtin*dt (main.f:613-632, 716-730, 820-826); dt is the
 * handle's.  Works on files the reference wrote.
 * mode IW_RESTART_EXACT: also restores the step counter, dt, the multistep
 * coefficients and the adaptive-step state from this library's extra
 * record, so the run continues bit for bit; IW_ERR_CONFIG if it is absent.
 * The handle's parameters stand: the reference also takes pr, ra and umax
 * from the file, which equal the namelist values when a run continues with
 * its own input.dat.  The output schedules (iw_set_animation,
 * iw_set_speclegen, iw_set_postp) are not in the file and stay as set on
 * the handle; the animation counter and Tdump restart from 0, as after the
 * reference's own restart (restart.f does not read them). */
int iw_read_restart(iw_handle *h, const char *path, int mode, double cdtin);

/* Replaces output.f:118-265 (plotf; main.f:543,607,1039): u, v, w and temp
 * in physical space, after t, nx ny nz ntot and the x, y, z grids.
 * iform 0: unformatted sequential (as the restart files), the fields as
 * REAL*4 over (nxpp, ny, nz); iform 1: formatted, 5e14.6 for reals and 5i10
 * for the dims.  The padding entries i = nx+1, nx+2 hold 0.  Asynchronous:
 * the transforms and the copies into a pinned host buffer are queued on the
 * handle's stream and the call returns; a host thread writes the file while
 * later steps run.  Call iw_wait_fields before reading the file.  The state
 * is not changed (the reference transforms it back, a projection the next
 * step's maxcalc round trip applies anyway). */
int iw_write_fields(iw_handle *h, const char *path, int iform);
/* Replaces the animation dumps of convec (solver.f:136-222, dtanim of the
 * &inputs namelist): with dtanim > 0, every iw_step whose time t is at least
 * dtanim past the last dump (Tdump, starting at 0 here) writes
 * dir/vortanimout_NNNNN.dat (NNNNN counts the dumps from 1): a list-directed
 * ZONE header, then x, z, u, w, temp, temp + rhomean(z) in physical space,
 * FORMAT (1x,6(F25.16,3x)), for every subdomain point and x index.  The rows
 * are those the reference reads: its y index is the value the preceding loop
 * leaves, ny+1, i.e. row 1 of the next z-plane, and past the last plane the
 * first rows of v, temp and un (COMMON /flow/ order).  Each dump also
 * appends its line to dir/animdump.log (solver.f:212-215).  Written like
 * iw_write_fields, by a host thread; iw_wait_fields waits for the last one.
 * dtanim <= 0 turns the dumps off.  Steps with dumps are not replayed from
 * graphs. */
int iw_set_animation(iw_handle *h, double dtanim, const char *dir);
/* Replaces main.f:905-910 with filtering.f:1110-1221 (speclegencalc): with
 * ncalclegspec > 0, every iw_step whose step number is a multiple of it
 * writes dir/speclegen<c><t>.dat for c = u, v, w, T after t += dt and before
 * the interface averaging: per subdomain and Legendre mode, the mean over x
 * of |a_k| in the x row at y index nyh.  Written like iw_write_fields, by a
 * host thread; iw_wait_fields waits for the last one.  IW_ERR_CONFIG for
 * ny = 1, where the reference's y index nyh = 0 lies outside the field.
 * ncalclegspec <= 0 turns the spectra off. */
int iw_set_speclegen(iw_handle *h, int ncalclegspec, const char *dir);

/* Replaces postp.f:9-70 with energycalc_postp (postp.f:415-732) and its
 * helpers (umeancalc, dudzmeancalc, dudymeancalc, perturbcalc): the TKE
 * budget of the current state.  e18 receives the values of one energy.dat
 * line, in its order: t - tstart, (t - tstart) brunt, tketot, u1tke, u2tke,
 * u3tke, prody, prodz, prod, bflux, epsilon, epssgs, epstot, chi, chisgs,
 * chitot, tkemean, tempvar; w18 those of energy_wake.dat.  u' is u minus its
 * x mean (0 at the bottom level); sums run over levels 2..nz; bflux carries
 * the reference's factor ra pr with ra = 0; the subgrid terms are 0 (no
 * subgrid model); the wake values are 0 but tkemean (the wake radii are
 * never set).  Either pointer may be NULL. */
int iw_postp(iw_handle *h, double *e18, double *w18);
/* main.f:935-936: with npostp > 0, every iw_step whose step number is a
 * multiple of npostp (after the interface averaging) appends one line to
 * dir/energy.dat, dir/energy_wake.dat and dir/wakescale.dat in the
 * reference's formats (headers written by the first line).  tstart is the
 * &mflags value the times are counted from.  npostp <= 0 turns it off. */
int iw_set_postp(iw_handle *h, int npostp, double tstart, const char *dir);
/* Waits for the last iw_write_fields to finish its file; returns its status
 * (IW_ERR_IO with the reason in iw_last_error() if the file failed). */
int iw_wait_fields(iw_handle *h);

/* Mode-1 internal wave initial condition plus seeded uniform noise in the
 * bottom 20% of the depth, transformed to spectral space (a new init: the
 * reference init.f sets zeros).  Deterministic for a given seed. */
int iw_init_mode1(iw_handle *h, double amplitude, double noise_amp,
                  uint64_t seed);

/* One complete time step of main.f:653-1066: maxcalc round trip, convec,
 * coefficient schedule, calcuvwt, t += dt, interface averaging.  The
 * coefficient schedule of main.f:700-856 is applied internally (fixed dt).
 * Failure detection (not in the reference): the first kernel of every step
 * flags a NaN or Inf in the state it reads, and a solve kernel whose bounded
 * wait for its tables gives up flags a timeout.  The flags reach the host
 * without a wait, so iw_step and iw_run return IW_ERR_NONFINITE (or
 * IW_ERR_TIMEOUT) from the first call after the flag has arrived, usually
 * one or two steps later, and then refuse to step; iw_sync and iw_diag wait
 * and report it at once.  A new state (iw_upload_state, iw_init_mode1,
 * iw_read_restart) clears the flags. */
int iw_step(iw_handle *h);
/* nsteps steps of main.f:653-1066.  With use_graph != 0, once the step is
 * invariant, steps are replayed from two captured CUDA graphs, one launch per
 * step. "Invariant" means: from step 4 with a fixed dt; no paddle forcing;
 * the filter every nspecfilterexp = 1 step; navgintrfc <= 1; profiling off.
 * Two graphs are needed because the history buffers alternate between two
 * arrangements.  Results are identical to the eager path.  Graphs are built
 * per call and freed before it returns. */
int iw_run(iw_handle *h, int nsteps, int use_graph);

/* Not in the reference.  Times the launch candidates of this handle's step on
 * its device and keeps the fastest for the following steps: y-tile width (2, 4
 * or 8 columns), the stage-A and stage-E variants (register-column or tiled)
 * and the solve variant (system-grouped CTAs with the tables staged in shared
 * memory, their block products on the FP64 pipes or on the FP64 tensor cores,
 * or one CTA per task of <= 4 right-hand sides).  Candidates run on the
 * handle's scratch fields; the state is not changed (the solver tables are
 * built if no step has built them yet).  The stage-A variants and the solve
 * variants 0 and 1 give the same bits; the stage-E variants and the
 * tensor-core products round differently.
 * choices (optional, 4 ints): the y-tile width; for stage A and stage E
 * 1 = register-column, 0 = tiled, -1 = not applicable (stage E also 2 =
 * tiled with the input tiles staged by bulk copies, N <= 64); the pressure
 * solve's variant (1 = system-grouped, 2 = system-grouped on the tensor cores,
 * N <= 40, 0 = per task; each solve role keeps its own fastest). */
int iw_autotune(iw_handle *h, int *choices);

/* Not in the reference.  Sets one launch choice of iw_autotune directly. */
#define IW_LAUNCH_YTILE 0   /* 0 (size heuristic), 2, 4 or 8 */
#define IW_LAUNCH_STAGE_A 1 /* -1 (size heuristic), 0 tiled, 1 register-column */
#define IW_LAUNCH_STAGE_E 2 /* as stage A, or 2: tiled, bulk-copied input tiles (N <= 33); 3: the same with
                               its z operators in the constant bank */
#define IW_LAUNCH_SOLVE 3   /* 1 system-grouped (default), 2 same on the FP64 tensor cores, 0 per task,
                               3 system-grouped with two rows per thread (u/v, w, rho; the pressure takes 1) */
/* one solve role's variant (values as IW_LAUNCH_SOLVE; -1 = the IW_LAUNCH_SOLVE choice) */
#define IW_LAUNCH_SOLVE_UV 4
#define IW_LAUNCH_SOLVE_W 5
#define IW_LAUNCH_SOLVE_RHO 6
#define IW_LAUNCH_SOLVE_PRESSURE 7
#define IW_LAUNCH_XROW_THREADS 8 /* threads per x-row CTA: 256 (0 = default) or 128 */
int iw_set_launch(iw_handle *h, int which, int value);

/* Not in the reference.  Reads one launch choice (the IW_LAUNCH_* ids), e.g.
 * the per-role solve variants iw_autotune kept. */
int iw_get_launch(iw_handle *h, int which, int *value);

/* Not in the reference (its main.f advances one run).  Advances n independent
 * runs of any sizes (separate handles on one device) by nsteps steps each.
 * Steps run eagerly until every member is invariant as for iw_run.  After
 * that, each step of the whole ensemble is one CUDA-graph launch, in which the
 * members are independent branches.  Each member's results are identical to
 * running it alone. */
int iw_ensemble_run(iw_handle *const *members, int n, int nsteps);
/* As iw_step but with caller-supplied coefficients (variable-dt restarts). */
int iw_step_coefs(iw_handle *h, const iw_coefs *c);
/* The values main.f keeps in COMMON /ab/ /bdf/ (comtimeadvance.h), dt and t
 * (COMMON /time/), set on the handle without stepping: convec_ reads fac1..3,
 * bdf1..3, dt and t, calcuvwt_ reads bdfv and dt.  A Fortran driver that
 * keeps main.f's own sequence (convec_, the coefficient updates of
 * main.f:700-856, calcuvwt_, t = t + dt, interface_avg3d_) calls this where
 * main.f assigns them. */
int iw_set_coefs(iw_handle *h, const iw_coefs *c, double t);

int iw_diag(iw_handle *h, iw_diag_out *out);
/* Mean (kx=ky=0) profiles of u, v, w, rho (4*nz doubles) copied to the host
 * buffer: the small per-step result a driver reads back. */
int iw_mean_profiles(iw_handle *h, double *host4nz);
int iw_sync(iw_handle *h);
/* raw device pointer of field f (0..3 = u,v,w,temp at level n) */
int iw_field_ptr(iw_handle *h, int f, void **dptr);
/* CUDA stream the handle works on (cudaStream_t) */
int iw_stream(iw_handle *h, void **stream);
/* bytes of device memory held by the handle */
int iw_device_bytes(iw_handle *h, size_t *bytes);

/* Batched vertical penalty solves (one Helmholtz system per (kx,ky)
 * column), the isolated-solve workload: lambda = kx^2+ky^2 + c, BCs by the
 * bc flags.  rhs/sol are complex columns [ncol][nz] as (re,im) pairs on the
 * device.  mode 0: FP64 factor + FP64 solve; 1: FP32 solve + one FP64
 * residual refinement.  The factors are built on the first call for a given
 * (c, ifbcbot, ifbctop) and kept. */
int iw_helm_solve_batched(iw_handle *h, const double *lam_dev, int ncol,
                          int ifbcbot, int ifbctop, const double *rhs_dev,
                          double *sol_dev, int mode);

/* Per-phase device time of the step, measured with CUDA events on the
 * handle's stream: enable=1 starts (and zeroes), 0 stops.  iw_profile_read
 * returns milliseconds and counts for 16 phases: 0 stageA, 1 y-inverse,
 * 2 x-row NL products, 3 y-forward, 4 wall BC term, 5 stageE, 6 pressure,
 * 7 u/v solve, 8 w solve, 9 rho solve, 10 interface averaging. */
int iw_profile(iw_handle *h, int enable);
int iw_profile_read(iw_handle *h, double *ms16, long *n16);

/* Make h the handle the Fortran-style entry points below act on. */
int iw_bind(iw_handle *h);

/* ---------------------------------------------------------------------- */
/* Drop-in replacements of the reference subroutines (Fortran calling      */
/* convention: every argument by reference; REAL = double).                 */
/* ---------------------------------------------------------------------- */

/* horfft.f:2-69.  In place on nk z-planes of (nxpp, ny) doubles.  is=-1:
 * physical -> spectral (x real-to-half-complex scaled 1/nx, then y complex
 * unscaled over the first nx/2 kx columns, everything scaled 1/ny).
 * is=+1: the inverse, unscaled.  Host array. */
void horfft_(double *b, const int *is, const int *nk);

/* derv.f:212-275: b = (2/zh(ks)) D a, per subdomain, whole field. Host. */
void dpdz_(const double *a, double *b);

/* filtering.f:811-983: Fourier (radial exponential) then Legendre modal
 * exponential filter of a spectral field, in place.  Host array. */
void filter_3dlegenfourier_(double *f, const int *ifourier, const int *ilegen,
                            const int *iout);

/* filtering.f:729-808: Legendre modal filter of one subdomain column. */
void filter_legenpen_(const double *fin, double *fout, const double *ybar,
                      const int *iprt, const int *ks);

/* penalty.f:714-775: adaptive interface averaging in physical space of a
 * spectral field, in place; ic returns the number of averaged points. */
void interface_avg3d_(double *f, int *ic);

/* penalty.f:162-251 (+ helmv_penalty 255-397, matrix_elmsetup 403-634,
 * band_lu.f:15-54): assemble the penalty system for epsilon and the BCs,
 * band-LU factor it and solve for the real and imaginary RHS.  rhsinr/rhsini
 * are multiplied by -epsilon in place, as in the reference. */
void penalty_main_(const double *epsilon, const int *ifuncreal,
                   const double *bcrbot, const double *bcibot,
                   const double *bcrtop, const double *bcitop,
                   const int *ifbcbot, const int *ifbctop, double *rhsinr,
                   double *rhsini, double *fr, double *fi);

/* band_lu.f:15-54: dense (nz x nz, column major) -> band storage, SGBTRF
 * (unblocked SGBTF2 path) and SGBTRS for xr and xi.  Solutions overwrite
 * xr/xi. */
void bandlu_solve_(const double *ain, double *xr, double *xi,
                   const int *ifuncreal);

/* No counterpart in the reference.  The work of bandlu_solve_ for callers that
 * must not allocate device memory while they run: a program whose device memory
 * belongs to its own pool sized at start-up (an extra cudaMalloc may fail or be
 * forbidden there), or a timing-critical loop that cannot take the device-wide
 * synchronisation of cudaFree.  It calls no cudaMalloc, cudaFree or other
 * allocating routine.
 *   ain_dev  device pointer, dense nz x nz matrix, column major, nz = nzloc*nsubd
 *            (kl = ku = nzloc, as in band_lu.f)
 *   x_dev    device pointer, nrhs (1 or 2) right-hand sides of nz values back to
 *            back; overwritten by the solutions
 *   stream   cudaStream_t to order the work on (NULL: the default stream); the
 *            call returns once the work is enqueued
 * Limits: nzloc in [2, 64], nsubd in [1, 64] and (3*nzloc+1)*nzloc*nsubd <=
 * 131072 (the band storage), which allows at most nz = 1600 (nzloc = 25,
 * nsubd = 64).  Other systems are refused with IW_ERR_CONFIG and a message in
 * iw_last_error().  No handle is needed; the current device is used.
 * Band storage, pivots and status sit in one fixed device array of about 1.06 MB
 * that each GPU loading this library holds until the process exits.  Every call
 * on a device uses that same array; each call rewrites all of it that it reads.
 * Calls that overlap on the GPU (other streams, other host threads) therefore
 * corrupt each other: order them, for example on one stream.
 * The first call on each device also does a one-time set-up (it looks up the
 * device address of the array); make that first call before any stream capture
 * begins.  The address is kept for the life of the process: do not call this
 * after a cudaDeviceReset of that device.  As in bandlu_solve_ and the
 * reference, a zero pivot is not reported. */
int iw_bandlu_solve_noalloc(const double *ain_dev, double *x_dev, int nzloc,
                            int nsubd, int nrhs, void *stream);

/* penalty.f:9-53: interior-subdomain Robin parameters for epsilon (kept in
 * the bound handle, used by the next penalty_main_). */
void penalty_setup_(const double *epsilon);

/* solver.f:6-514 on the bound handle's device state. */
void convec_(const int *istep, const int *istart, const int *ispecfilternl);
/* calcuvwt*.f on the bound handle's device state; cpenspecfilter is a
 * Fortran LOGICAL (4-byte int, nonzero = .true.). */
void calcuvwt_(const int *izmode, const int *ispecfilter, const int *irelax,
               const int *cpenspecfilter);

/* multistep.f:7-89: variable-step AB3 / BDF3 coefficients. */
double abvar1_(const double *dt1, const double *dt2, const double *dt3);
double abvar2_(const double *dt1, const double *dt2, const double *dt3);
double abvar3_(const double *dt1, const double *dt2, const double *dt3);
double bdfvarv_(const double *dt1, const double *dt2, const double *dt3);
double bdfvar1_(const double *dt1, const double *dt2, const double *dt3);
double bdfvar2_(const double *dt1, const double *dt2, const double *dt3);
double bdfvar3_(const double *dt1, const double *dt2, const double *dt3);

/* various.f:892-982: the adaptive time-step rule maxcalc applies at the start
 * of every step, as a pure host function (the handle API applies it itself
 * when imaxcalc = 1).  In: the CFL numbers cflx, cflz of the fields at the
 * start of the step, the time t, the current step dt and the wave frequency
 * xomega (main.f:341-346).  Returns 1 and sets *dt_new = dt / cdt and *cdt when
 * the step changes, else 0 and leaves both untouched.  The step changes when
 * int(t / dt) > 20 and cflz > 0.7, cflz < 0.1 or cflx > 0.16; cdt = 1.25 if
 * cflz > 0.7 or cflx > 0.16, else max(0.8, dt / Tlim) with
 * Tlim = 2 pi / (50 xomega).  The step count is taken from t = 0: the
 * reference's Tso (various.f:918,924) is a local without SAVE that is read
 * before it is written, and its own recorded run (dtchange.dat) changes dt
 * exactly when int(t / dt) > 20. */
int iw_dt_rule(double cflx, double cflz, double t, double dt, double xomega,
               double *dt_new, double *cdt);

#ifdef __cplusplus
}
#endif
#endif /* IW_B200_H */
