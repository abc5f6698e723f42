/*
 * sac_gpu.h -- C-ABI of the B200 perturbation-MHD hot path (libsacgpu.so).
 *
 * The entry points replace the Fortran call surface of the reference's hot path
 * (drewleonard42/SAC, files cited relative to the project root):
 *
 *   sac_create          physini + the method part of readparameters   src/vacphys.mhd0.t:9, src/vacio.t:246-527
 *   sac_set_grid        setixGixMix + gridsetup1 (dx, dvolume)         src/vacio.t:786-841, src/vacgrid.t:556-661
 *   sac_set_boundaries  boundsetup (default or user regions, pairing)   src/vacgrid.t:9-160
 *   sac_upload          host w(ixG^T,nw) -> resident device state      (the COMMON w of program vac, src/vac.t:12)
 *   sac_download        resident device state -> host w                (savefile, src/vacio.t:901)
 *   sac_getboundary     getboundary(t,1,nw,1,ndim,w)                   src/vacgrid.t:195-512
 *                       (with keeppositive first when smallfix)        src/vacphys.t.mhd:8-49
 *   sac_getdt           vac.t dt block: getdt_courant+getdt+getdt_special src/vac.t:60-70,641-699;
 *                                                                      src/vacphys.mhd0.t:83; src/vacusr.f:1403
 *   sac_advect          advect(method,ixG^L,iws,idim^LIM,w1,w)         src/vac.t:364-487
 *   sac_diag            getdivb + volume means of savefilelog_default  src/vacphys.mhd0.t:106; src/vacio.t:1094
 *                       + nerror(toosmallp_) of keeppositive           src/vac.t:117-136
 *
 * Conventions
 *   - Arrays crossing the ABI are Fortran order: w(ix1,ix2,ix3,iw), x1 fastest,
 *     one contiguous block per variable (SoA), ixGlo=1, exactly the reference's
 *     COMMON/stack layout (src/vacdef.t:18-23, src/vac.t:12).
 *   - Strings are Fortran CHARACTER*10 blank-padded (no NUL) where marked
 *     "f10"; method names may also be NUL-terminated C strings.
 *   - Every call returns a status; nothing exits or traps.  The Fortran shim maps
 *     a non-zero status to die() (src/vacio.t:1152).  sac_last_error() holds the text.
 *   - One context per host thread; a context is not re-entrant.
 *   - The state stays resident on the device between calls; w1/w2/w3 of the
 *     reference's advect are device-internal scratch.
 */
#ifndef SAC_GPU_H
#define SAC_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

#define SAC_LENTYPE 10 /* CHARACTER*^LENTYPE, src/vacpp.pl:156 */
#define SAC_NHIB 10    /* nhiB, src/vacdef.t:34 */
#define SAC_NWMAX 13   /* nw for -d=33 -p=mhd, src/vacpar.t.mhd:9-13 */

typedef int sac_status;
#define SAC_OK 0
#define SAC_ERR_ARG 1         /* bad argument (die() in the reference) */
#define SAC_ERR_STATE 2       /* call out of order (grid/boundaries/state not set) */
#define SAC_ERR_CUDA 3        /* CUDA runtime error */
#define SAC_ERR_NOMEM 4       /* device allocation failed */
#define SAC_ERR_UNSUPPORTED 5 /* option outside the implemented path */
#define SAC_ERR_NONFINITE 6   /* NaN/Inf met in a reduction */
#define SAC_ERR_TIMEOUT 7     /* a bounded device wait ran out */
#define SAC_ERR_NODEVICE 8    /* no usable CUDA device */

/* Storage precision of the perturbed variables (the background is always FP64). */
#define SAC_PREC_FP64 0
#define SAC_PREC_FP32 1

/* User modules: the specialsource/getdt_special plug-in of vacusr.t.
 *   SAC_USR_NONE       no special sources
 *   SAC_USR_VISCOSITY  hyperdiffusion only, no dt limit     sac/src/vacusr.t.stuart:46-94
 *   SAC_USR_SLOG       gravity + hyperdiffusion + Gaussian vortex driver,
 *                      dt limits from viscosity and gravity src/vacusr.f:1255-1421
 *   SAC_USR_GRAVVISC   gravity + hyperdiffusion, both dt limits (vacusr.gravity.t +
 *                      vacusr.viscosity.t without a driver)
 *   SAC_USR_STRAT      gravity + hyperdiffusion + a vertical-velocity driver near the
 *                      lower x1 boundary (stratified-atmosphere workload)
 *   SAC_USR_TUBE       gravity + hyperdiffusion + a horizontal (x2) velocity driver near
 *                      the lower x1 boundary (2D flux-tube workload)          */
#define SAC_USR_NONE 0
#define SAC_USR_VISCOSITY 1
#define SAC_USR_SLOG 2
#define SAC_USR_GRAVVISC 3
#define SAC_USR_STRAT 4
#define SAC_USR_TUBE 5

typedef struct sac_params {
  /* equation parameters eqpar(1:neqpar+nspecialpar), src/vacpar.t.mhd:26,
   * src/vacusrpar.f:3-6 */
  double gamma;   /* eqpar(gamma_) */
  double eta;     /* eqpar(eta_): 0, or a constant resistivity > 0 (addsource_res2, or
                   * addsource_res1 with compactres, and getdt_res, src/vacphys.mhdres.t);
                   * eta < 0 (a user specialeta) is SAC_ERR_UNSUPPORTED */
  double grav[3]; /* eqpar(grav1_..grav3_) */
  double nu;      /* eqpar(nu_): hyperdiffusion on when |nu|>smalldouble */
  /* &paramlist, src/vacio.t:47 */
  double courantpar;
  double dtpar;
  double dtdiffpar;
  int dtcantgrow;
  /* &methodlist, src/vacio.t:33 */
  char typeadvance[SAC_LENTYPE + 1]; /* onestep|twostep|threestep|fourstep|sterck|jameson */
  char typepred[SAC_LENTYPE + 1];    /* predictor of 'twostep': 'nul' or 'cd4' */
  int sourceunsplit;                 /* sources added inside centdiff4 (par/DEFAULT:44) */
  int divbfix;                       /* Powell div B source (addsource_divb, src/vacphys.mhd0.t:263-297),
                                      * added when ndim > 1 and sourceunsplit.  par/DEFAULT:46 sets T;
                                      * sac_default_params leaves 0, as the reference's 3D pars do */
  /* plug-in */
  int user;            /* SAC_USR_* */
  /* driver parameters.  SAC_USR_STRAT: [0]=amplitude A, [1]=omega, [2],[3]=driver
   * centre in x2,x3, [4]=horizontal Gaussian width, [5]=x1 centre, [6]=x1 width.
   * SAC_USR_TUBE: [0]=A, [1]=omega, [2]=x1 centre, [3]=x1 Gaussian width,
   * [4]=x2 centre, [5]=x2 width.  Unused for the other modules. */
  double userpar[16];
  int alias_nu_grav3;  /* reproduce eqpar(nu_)==eqpar(grav3_) (src/vacusrpar.f:4-5) */
  int precision;       /* SAC_PREC_FP64 | SAC_PREC_FP32 */
  int device;          /* CUDA ordinal (ignored by the CPU oracle) */
  /* &methodlist smallfix and its floors, src/vacio.t:44-45 (defaults :99-101 and
   * par/DEFAULT:54).  With smallfix set, every boundary fill first runs
   * keeppositive (src/vacphys.t.mhd:8-49) on the mesh: where rho'+rhob < smallrho the
   * cell gets the vacuum state (m=0, rho'=vacuumrho-rhob, e' from smallp and b');
   * then, if any thermal pressure is below max(0,smallp), nerror(toosmallp_) counts
   * the fill and, for smallp > 0, e' is rebuilt from max(p,smallp) on the whole
   * mesh.  The batched contexts reject smallfix with SAC_ERR_UNSUPPORTED. */
  int smallfix;
  double smallp;       /* default -1 */
  double smallrho;     /* default -1 */
  double vacuumrho;    /* default -1 */
  /* &methodlist compactres (par/DEFAULT:57, F): the resistive source in its compact
   * form addsource_res1 (src/vacphys.mhdres.t:96-220), eta times the 3-point
   * Laplacian of B into b and e plus eta J^2 into e, instead of addsource_res2.  The
   * batched contexts reject it with SAC_ERR_UNSUPPORTED. */
  int compactres;
} sac_params;

typedef struct sac_diag_out {
  double wmean[SAC_NWMAX]; /* dvolume-weighted means over the mesh (savefilelog_default) */
  double divb_l2;          /* sqrt(mean (div B)^2) over the mesh, 4th-order getdivb stencil */
  double divb_linf;        /* max |div B| over the mesh */
  double maxviscoef;       /* running max of nu over the current step (setnu) */
  double ctot[3];          /* last c_tot per dimension used by setnu */
  int nonfinite;           /* 1 if a NaN/Inf was seen in the mesh */
  /* keeppositive's error record (smallfix): nerror(toosmallp_), the fills whose
   * thermal pressure went below max(0,smallp); the step number of the first such
   * fill (the it last passed to sac_getdt or sac_advect, 0 before either) and the
   * minimum pressure over the mesh at that fill, which the reference prints then
   * (src/vacphys.t.mhd:34-41) */
  int nerror_toosmallp;
  int toosmallp_it;
  double toosmallp_min;
} sac_diag_out;

typedef struct sac_ctx sac_ctx;

/* Fill p with the reference's defaults (par/DEFAULT + physini). */
void sac_default_params(sac_params* p);

sac_status sac_create(const sac_params* p, sac_ctx** out);

/* ndim, ndir: -d=NdimNdir.  ixGhi[0..2]: grid extents with ghosts (ixGlo=1; unused
 * dims 1).  ixM[0..5]: ixMmin1..3, ixMmax1..3 (1-based).  x: x(ixG^T,ndim) Fortran
 * order; when fullgridini is 0 only the mesh part is read and the ghost coordinates
 * are extrapolated as gridsetup1 does. */
sac_status sac_set_grid(sac_ctx* c, int ndim, int ndir, const int ixGhi[3], const int ixM[6],
                        const double* x, int fullgridini);

/* boundsetup (src/vacgrid.t:9-160) with &boundlist's nB, typeB, ixB^LIM, idimB,
 * upperB and ipairB (src/vacio.t:46, src/vacdef.t:107-111).
 *   typeB  CHARACTER*10 typeB(nw,nB) (f10, blank padded).
 *   ixB    NULL: the default regions, nB = 2*ndim, iB=2*idim-1 (lower) / 2*idim
 *          (upper), each a full dixB-deep ghost slab.  Otherwise the user's
 *          regions: ixBmin(1:ndim,1:nB) followed by ixBmax(1:ndim,1:nB) (1-based,
 *          Fortran order), with idimB(1:nB) in 1..ndim and upperB(1:nB) 0/1 (both
 *          required then).  Each region must lie inside the grid (SAC_ERR_ARG, as
 *          boundsetup's die) and in the ghost layers along its idimB; regions
 *          2*idim-1 and 2*idim must be the lower and upper boundaries of dimension
 *          idim, which gradient4, gradient1 and setnu read; regions beyond 2*ndim
 *          are free (up to nhiB = 10).  getboundary fills the regions in order,
 *          later ones overwriting earlier ones where they overlap.
 *   ipairB NULL or ipairB(1:nB), 0 = pair automatically: the periodic regions of the
 *          same idimB, opposite upperB and equal extent. */
sac_status sac_set_boundaries(sac_ctx* c, int nB, const char* typeB, const int* ixB, const int* idimB,
                              const int* upperB, const int* ipairB);

/* w is always the host's FP64 w(ixG^T,nw).  There is no per-call storage mode:
 * the precision of the resident perturbed variables is the context's
 * sac_params.precision, fixed at sac_create because the FP32 path's arrays and
 * kernels are chosen then; upload rounds to it and download widens from it. */
sac_status sac_upload(sac_ctx* c, const double* w);
sac_status sac_download(sac_ctx* c, double* w);
sac_status sac_getboundary(sac_ctx* c, double t);

/* On return *dt holds the step of the dt block of the main loop, src/vac.t:61-70
 * (dtpar, getdt_courant, getdt with getdt_res for eta > 0, getdt_special,
 * dtcantgrow).  it is the step number. */
sac_status sac_getdt(sac_ctx* c, double* dt, int it);

/* method: typefull1 ('cd4' | 'source' | 'nul'); iws: iws(1:nw+1), iws(nw+1)=count,
 * or NULL for all advanced variables.  The unsplit sources are the user module's
 * (gravity, hyperdiffusion, driver), then addsource's resistive (eta > 0) and
 * Powell (divbfix, ndim > 1) terms. */
sac_status sac_advect(sac_ctx* c, const char* method, const int* iws, int idimmin, int idimmax,
                      double dt, double t, int it);

sac_status sac_diag(sac_ctx* c, sac_diag_out* out);
sac_status sac_synchronize(sac_ctx* c);
const char* sac_last_error(const sac_ctx* c);
void sac_destroy(sac_ctx* c);

/* ---- library extensions: no counterpart in the reference ------------------
 * Stream selection lets a host run the path on its own CUDA stream; profiling
 * brackets every kernel launch with CUDA events on that stream. */
#define SAC_K_STAGE 0   /* k_update: the per-cell stage update */
#define SAC_K_PREP 1    /* k_face: derived fields, fluxes, c_tot */
#define SAC_K_BOUND 2   /* k_bound: ghost-cell resolve */
#define SAC_K_COURANT 3 /* getdt_courant reduction */
#define SAC_K_OTHER 4   /* conversions, copies and RK combinations */
#define SAC_K_NU 5      /* k_nu: setnu face ratios */
#define SAC_K_COUNT 6
sac_status sac_set_stream(sac_ctx* c, void* cuda_stream); /* NULL: the context's own stream */
void* sac_get_stream(const sac_ctx* c);
sac_status sac_profile(sac_ctx* c, int enable);
/* synchronises, then returns the summed event time and launch count of kernel
 * class `kernel` since the last reset (reset != 0 clears after reading) */
sac_status sac_profile_read(sac_ctx* c, int kernel, double* total_ms, long* launches, int reset);
long sac_kernel_launches(const sac_ctx* c);

/* ---- getdt that allocates nothing (library extension; no reference counterpart) ----
 * For callers that cannot allocate device memory where they need dt, such as a
 * host that gives the whole device to its own pre-sized pool.  Same result and
 * side effects as sac_getdt; like sac_getdt it launches its reductions on the
 * context's stream, copies the maximum back and waits for that stream, so it is
 * an ordinary host call (not for use inside a host callback).  Its getdt_courant reduction
 * runs as a deterministic two-pass block reduction whose scratch (8192 partial
 * maxima and the result, 64 KB) is a file-scope device array of the library, held by
 * every GPU that loads the library until the process exits; the call makes no
 * cudaMalloc/cudaFree or other allocating call.
 *   - Limit: meshes of at most SAC_STATIC_MAX_CELLS cells; a larger mesh returns
 *     SAC_ERR_UNSUPPORTED with the sizes in sac_last_error (use sac_getdt there).
 *   - The scratch is one per device, shared by every context on it: calls that
 *     overlap in time (other host threads, other streams) race on it.
 *   - The first call on a device also looks up the scratch's device address
 *     (cudaGetSymbolAddress), once per device, and keeps it for the life of the
 *     process: the device's primary context (the runtime's, which every context
 *     of this library uses) must not be reset (cudaDeviceReset) while the library
 *     is loaded, or the kept address no longer names the scratch.
 *   - With profiling on, its two launches count under SAC_K_COURANT, as the
 *     reduction of sac_getdt does.
 *   - Nothing in the scratch has to start at zero: each slot that is read was
 *     written earlier in the same call. */
#define SAC_STATIC_MAX_CELLS 33554432L
sac_status sac_getdt_static(sac_ctx* c, double* dt, int it);

/* ---- many independent grids (library extension, no Fortran counterpart) ----
 * A batch advances ninst uneven 1D/2D problems together, each with its own dt,
 * with typeadvance='fourstep' (the RK4 step of src/vac.t:439-455) and the dt
 * block of src/vac.t:60-70 per instance.  Every instance is a separate program
 * vac run: the same parameters (sac_params, shared), its own mesh nx(ndim) with
 * two ghost layers per side, its own coordinates and state.  Boundary types that
 * store ghost values (fixed, fixed1, grad1) and the Slog driver are not available
 * here (SAC_ERR_UNSUPPORTED), nor is a user resistivity (eta < 0); constant
 * resistivity (eta > 0) and the Powell source (divbfix, ndim = 2) are.  The
 * Gaussian drivers (strat, tube) take their amplitude and frequency per instance
 * (sac_batch_set_driver).
 *
 * Host arrays are the instances' Fortran-order blocks one after another:
 *   x: instance i contributes x(ixG^T,ndim), w: instance i contributes w(ixG^T,nw),
 *   ixG^T = (nx1+4)[*(nx2+4)].
 * group_cells bounds the cells of the per-stage intermediates (0: 2^26): the
 * instances are processed in consecutive groups of at most that many cells.
 * The step is recorded once as a CUDA graph on the batch's own stream and
 * replayed by sac_batch_advance; nothing in it synchronises with the host. */
typedef struct sac_batch sac_batch;
sac_status sac_batch_create(const sac_params* p, int ndim, int ndir, int ninst, const int* nx, long group_cells,
                            sac_batch** out);
sac_status sac_batch_set_grid(sac_batch* b, const double* x);
/* typeB f10 [nw][2*ndim], the same for every instance */
sac_status sac_batch_set_boundaries(sac_batch* b, const char* typeB);
sac_status sac_batch_upload(sac_batch* b, const double* w);
sac_status sac_batch_download(sac_batch* b, double* w);
/* the same for instances i0..i0+n-1 only (w holds just their blocks) */
sac_status sac_batch_upload_range(sac_batch* b, int i0, int n, const double* w);
sac_status sac_batch_download_range(sac_batch* b, int i0, int n, double* w);
sac_status sac_batch_getboundary(sac_batch* b);
/* enqueue nsteps RK4 steps of every instance (asynchronous) */
sac_status sac_batch_advance(sac_batch* b, int nsteps);
/* synchronises; per instance t, the last dt and the step count (each may be NULL);
 * SAC_ERR_NONFINITE when an instance met NaN/Inf in its dt reductions */
sac_status sac_batch_state(sac_batch* b, double* t, double* dt, int* it);
sac_status sac_batch_synchronize(sac_batch* b);
void* sac_batch_get_stream(const sac_batch* b);
/* time the update pass for each candidate tile shape on this batch and keep the
 * fastest; tile_xy[2] and ms (per update pass) receive the choice (may be NULL);
 * then time one whole stage in both stage forms (below) and keep the faster */
sac_status sac_batch_tune(sac_batch* b, int* tile_xy, double* ms);
/* Stage form.  By default each RK stage is three passes (face, setnu, update)
 * through device-wide intermediates.  For 2D instances with the default sources
 * (no Powell or resistive term) it can instead be one fused kernel per tile of
 * TX x TY mesh cells that computes the fluxes, setnu's quotients and the update
 * in shared memory (shapes: 0 = 32 x 8, 1 = 16 x 8); the results are the same
 * bit for bit.  sac_batch_tune times both forms on the batch and keeps the
 * faster; sac_batch_set_stage chooses one (SAC_ERR_UNSUPPORTED where the fused
 * form does not apply); sac_batch_get_stage reports the form and the tuner's
 * times of one stage (ms). */
sac_status sac_batch_set_stage(sac_batch* b, int fused, int shape);
sac_status sac_batch_get_stage(const sac_batch* b, int* fused, int* shape, double* ms_three, double* ms_fused);
/* FP64 and FP32-perturbation instances advanced together.  After
 * sac_batch_join(lead, partner), sac_batch_advance(lead, n) advances the
 * instances of both batches in one CUDA graph per step, each instance with its
 * own dt.  lead holds FP64 instances, partner FP32 ones, with the same parameters
 * (all but the precision), ndim = 2, ndir and device; both must have had their
 * first boundary fill; both take the fused stage in the lead's tile shape.  The
 * graph has one of two forms:
 *   0  joint kernels: every kernel of the RK4 step (getdt_courant, the dt block,
 *      c_tot, the fused stage, the boundary fill) is one persistent launch over
 *      the tiles of both batches;
 *   1  two branches: each batch's own kernels, the partner's on its own stream
 *      beside the lead's.
 * sac_batch_join times one RK stage in each form and keeps the faster;
 * sac_batch_set_join_form overrides it and sac_batch_get_join reports the form
 * (-1 when b leads no pair) and the two times (ms).  The FP64 instances advance
 * bit for bit as in a batch of their own in both forms.  In form 0 the FP32
 * instances compute without FMA contraction (the FP64 units' rounding rules), so
 * they may differ in the last bits from an FP32 batch advanced alone.  While
 * joined, the partner's work runs on the lead's stream (sac_batch_get_stream
 * returns it), and sac_batch_advance, sac_batch_tune, sac_batch_set_stage,
 * sac_batch_set_grid and sac_batch_set_boundaries of either batch are
 * SAC_ERR_STATE, except advancing the lead; uploads, downloads, the state,
 * drivers, times and packing work on each batch as before.
 * sac_batch_unjoin(lead), or destroying either batch, ends the join. */
sac_status sac_batch_join(sac_batch* lead, sac_batch* partner);
sac_status sac_batch_unjoin(sac_batch* lead);
sac_status sac_batch_set_join_form(sac_batch* lead, int form);
sac_status sac_batch_get_join(const sac_batch* lead, int* form, double* ms_joint, double* ms_forked);
/* per-instance driver amplitude and angular frequency of the Gaussian velocity
 * drivers (users SAC_USR_STRAT and SAC_USR_TUBE, tdep = sin(omega t)); the
 * defaults are userpar[0] and userpar[1].  Either array may be NULL. */
sac_status sac_batch_set_driver(sac_batch* b, const double* A, const double* omega);
/* per-instance time and step counter (either may be NULL) */
sac_status sac_batch_set_time(sac_batch* b, const double* t, const int* it);
/* per-instance end time, the reference's tmaxexact (src/vac.t:82): dt is clipped
 * to tmax - t + smalldouble, and an instance that reached tmax takes dt = 0
 * steps that leave its state and step counter untouched.  tmax <= 0: no limit. */
sac_status sac_batch_set_tmax(sac_batch* b, const double* tmax);
/* mesh cells over all instances (ghosts excluded) */
long sac_batch_mesh_cells(const sac_batch* b);
/* Packed mesh copies between the resident state and a DEVICE buffer, enqueued on
 * the batch stream: instance i contributes np*mesh_i values, variable-major
 * (rho, m.., e, b..), x1 fastest, ghosts excluded, in instance order.  dtype
 * SAC_PACK_F32 | SAC_PACK_BF16 | SAC_PACK_F64.  After a scatter, call
 * sac_batch_getboundary to refill the ghost cells. */
#define SAC_PACK_F32 0
#define SAC_PACK_BF16 1
#define SAC_PACK_F64 2
sac_status sac_batch_gather(sac_batch* b, void* dev, int dtype);
sac_status sac_batch_scatter(sac_batch* b, const void* dev, int dtype);
const char* sac_batch_last_error(const sac_batch* b);
void sac_batch_destroy(sac_batch* b);

#ifdef __cplusplus
}
#endif
#endif /* SAC_GPU_H */
