/*
 * dsem_gpu.h -- C-ABI of the B200 implementation of DSEM's right-hand side
 * and low-storage Runge-Kutta stage (FP64, sm_100a).
 *
 * The library replaces the body of DSEM's
 *     SUBROUTINE tstep(time,dt,d,ngrid,mrtr,nmort,resid)        (src/tstep.f90:12-120)
 * called from the time loop at src/3DDriver_parfmdf.f90:466.  DSEM's Fortran
 * keeps the mesh, the case input and the time loop; it packs the geometry of
 * TYPE(domain) d(:) and TYPE(mortar) mrtr(:) (src/paraFMDF/initializationsc2.f90:50-215)
 * once, after the setup at src/3DDriver_parfmdf.f90:307, and calls dsem_create.
 * From then on all element and interface state stays resident in HBM.
 *
 * Conventions
 *  - Plain C types only; host arrays are caller-owned and read (or written)
 *    only during the call.  Device state is library-owned.
 *  - Every function returns 0 (DSEM_OK) or a negative DSEM_ERR_* code; the
 *    text of the last error is available from dsem_last_error().  Nothing
 *    exits or aborts.
 *  - One context per host thread; calls on a context are not re-entrant and
 *    are synchronous on return (one CUDA stream per context).
 *  - Per-element arrays use DSEM's Fortran column-major layout padded to the
 *    caller's extent ldx (the `nx` of size.f90): element e, variable v,
 *    point (n,m,l) (0-based) sits at  n + ldx*(m + ldx*(l + ldx*(v + 5*e))).
 */
#ifndef DSEM_GPU_H
#define DSEM_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

#define DSEM_OK 0
#define DSEM_ERR_INVALID_ARG (-1)
#define DSEM_ERR_CUDA (-2)
#define DSEM_ERR_NONFINITE (-3)   /* mirrors the NaN/Inf abort of 3DDriver_parfmdf.f90:489-499 */
#define DSEM_ERR_TIMEOUT (-4)     /* a bounded device-side wait gave up */
#define DSEM_ERR_UNSUPPORTED (-5) /* mesh feature outside the implemented path */
#define DSEM_ERR_NOMEM (-6)

/* Integers per mortar in dsem_mesh_desc.mortar, mirroring TYPE(mortar)
 * (src/paraFMDF/initializationsc2.f90:193-215):
 *  [0] id(1)  master element (1-based)     [1] id(2) slave element (1-based)
 *  [2] iface(1) (1..6)                     [3] iface(2)
 *  [4] len(1,1) [5] len(2,1) [6] len(1,2) [7] len(2,2)
 *  [8] lenmortar(1) [9] lenmortar(2)       [10] orient (Edge_Mappings: 0..7)
 *  [11] sign  [12] nsign                   [13..16] conforming(1,1),(2,1),(1,2),(2,2) as 0/1 */
#define DSEM_MORTAR_INTS 17

typedef struct dsem_ctx dsem_ctx; /* opaque, owned by the library */

/* Geometry packed from d(:) and mrtr(:).  ldx is the padded extent of the
 * caller's arrays (>= ncg+1 of every element). */
typedef struct {
  int ngrid;             /* number of elements (ngrid in tstep)                        */
  int nmort;             /* number of mortars (nmort in tstep)                         */
  int ldx;               /* padded extent nx of the caller's per-element arrays        */
  const int *ncg;        /* [ngrid][3] Gauss points per direction, d%ncg               */
  const double *jacob;   /* [ngrid][ldx^3]       d%jacob   (1/J at Gauss points)       */
  const double *gmetg;   /* [ngrid][ldx^3][3][3] d%gmetg(3,3,nx,ny,nz) (grad xi)       */
  const double *gmet;    /* [ngrid][ldx^3][3][3] d%gmet(3,3,nx,ny,nz) (J grad xi on the
                            staggered grids; row i on grid i)                          */
  const int *mortar;     /* [nmort][DSEM_MORTAR_INTS]                                   */
  const double *n_hat;   /* [nmort][ldx][ldx][3]  mrtr%n_hat(3,nmax,nmax)               */
  const double *norm;    /* [nmort][ldx][ldx]     mrtr%norm(nmax,nmax)                  */
  const int *bcond;      /* [ngrid][6] d%bcond as DSEM_BC_* codes; read for the master
                            faces of boundary mortars (id(2) = 0). NULL: no boundary   */
} dsem_mesh_desc;

/* d%bcond values of faces without a neighbour (boundary_flux / DirichletBC /
 * Vis_Neumann in caseFiles/tgv/BackstepProblem-stoch.f90:1602-1729). */
#define DSEM_BC_INTERFACE 0
#define DSEM_BC_WALLADIAB 1 /* 'walladiab': wallbc_Inv, set_adiabatic_wall, wall_vis_flux   */
#define DSEM_BC_WALLISOTH 2 /* 'wallisoth': wallbc_isoth (osher), set_isothermal_wall        */
#define DSEM_BC_INFLOW 3    /* 'inflow':  inflow_specAll, boundary_values, boundary_vis_flux */
#define DSEM_BC_OUTFLOW 4   /* 'outflow': outflow_specAll, boundary_values, boundary_vis_flux */

/* Physics and time-integration parameters (MODULE physics, input_data, rk_coefs). */
typedef struct {
  double gamma, re, pr, mach; /* NS_data.f90:51-201                                    */
  double cmu, mumax;          /* entropy-viscosity coefficients                        */
  int shock;                  /* 1: entropy viscosity (tstep.f90:36-38); 3: also the
                                 Ducros sensor (input keyword `ducrosSens`, logical
                                 ducrosSensor: input_lib.f90:166, 442-443; applied at
                                 EViscosity_GL.f90:84)                                 */
  int iord;                   /* rkcoefs order: 3 (3 stages) or 4 (5 stages)           */
} dsem_phys;

/* Creates a context on the current CUDA device and copies the geometry to HBM.
 * Replaces nothing in DSEM itself: it is the one-time upload that precedes the
 * time loop (3DDriver_parfmdf.f90:307). */
int dsem_create(const dsem_mesh_desc *mesh, const dsem_phys *phys, dsem_ctx **out);
/* dsem_create for meshes whose axis-aligned elements carry rounding noise in their
 * metrics: DSEM's trilinear map (grad_hex8_map, GeomLib3D.f90) leaves off-diagonal
 * entries of ~1e-14 relative on most box sizes (28^3 and up), which send every element
 * to the general-metric volume kernel (2.2x slower per element at p = 8).  Entries of a
 * point whose magnitude is at most metric_snap times the point's largest diagonal entry
 * count as zero, so such elements take the diagonal kernel; the right-hand side then
 * differs from DSEM's by about metric_snap relative.  metric_snap = 0 is dsem_create;
 * values must lie in [0, 1e-6). */
int dsem_create_snapped(const dsem_mesh_desc *mesh, const dsem_phys *phys, double metric_snap, dsem_ctx **out);
void dsem_destroy(dsem_ctx *ctx);
const char *dsem_last_error(const dsem_ctx *ctx); /* ctx may be NULL (creation errors) */

/* J*Q state in/out (d%Q, stored as Q/jacob, 3DDriver_parfmdf.f90:290-300). */
int dsem_upload_q(dsem_ctx *ctx, const double *JQ, int ldx);
int dsem_download_q(dsem_ctx *ctx, double *JQ, int ldx);

/* Replaces the body of tstep (tstep.f90:36-116), nsteps times:
 * entropy viscosity (if enabled), g_Q = 0, kord stages of Fluxes + update.
 * dt is the global step (delta_t(1)).  Returns DSEM_ERR_NONFINITE when the
 * stage residual max|Qt| is not finite (checked once per dsem_step call). */
int dsem_step(dsem_ctx *ctx, double time, double dt, int nsteps);

/* One Runge-Kutta stage kk (1-based).  kk==1 also evaluates the entropy
 * viscosity and zeroes g_Q.  Qt (may be NULL) receives the stage Qt. */
int dsem_stage(dsem_ctx *ctx, double time, double dt, int kk, double *Qt, int ldx);

/* Parity hook: one evaluation of Fluxes (fluxesH_newa.f90:17) and the flux
 * divergence Qt (updatea.f90:100-113) without the update. */
int dsem_rhs(dsem_ctx *ctx, double tk, double *Qt, int ldx);

/* Diagnostics of the current state, the do_user_stuff / energydissipation
 * analogue (caseFiles/tgv/BackstepProblem-stoch.f90:463-709,
 * Energydissipation/energydissipation.f90:2-89):
 *   ke   = 1/2 <u.u> over the periodic [0,2pi]^3 box          (fort.22)
 *   dkdt = (ke_prev - ke)/dt, ke_prev = 0 when first != 0     (fort.23)
 *   eps  = 100 <|w|^2>/Re from the last stage's gradients      (dissipated) */
int dsem_diag(dsem_ctx *ctx, double dt, int first, double *ke, double *dkdt, double *eps);

/* Entropy-viscosity coefficient muhg at Gauss points (ldx layout, one field). */
int dsem_get_muhg(dsem_ctx *ctx, double *mu, int ldx);

/* Device time of the last dsem_step call, and the number of kernel launches
 * it made (for benchmarking). */
int dsem_last_timing(const dsem_ctx *ctx, double *ms, long long *launches);

/* Benchmark hook (no DSEM counterpart): times reps evaluations of each
 * kernel of a right-hand side with CUDA events on the context's stream and
 * returns the mean milliseconds per evaluation in ms[4] = {inviscid face,
 * volume, viscous face, divergence + update}.  The state is left unchanged.
 * The kernels are those dsem_step runs: where every element face is one side
 * of a conforming mortar, the update kernel averages the viscous face fluxes
 * itself, so ms[2] is then about zero and ms[3] includes that average. */
int dsem_profile_rhs(dsem_ctx *ctx, int reps, double *ms);

/* Static Smagorinsky LES (tstep.f90:40-43, turbulence/staticSmago/staticSmag.f90):
 * at the start of every step the subgrid viscosity
 *   nu_t = Re (C_s delta_g)^2 |S|, clipped to [0, numax],
 * is formed at Gauss points from the gradients of the previous step's last
 * stage (zero before the first), prolonged to the Lobatto grids (negatives
 * set to 0) and added to the viscosity as amu = 1 + nu_t rho (+ mu_EV)
 * (Vis_Fluxes_new.f90:123-125).  cs = 0 turns it off.  DSEM's input keywords:
 * `smagorinsky`, C_s, numax; its shock and density sensors are not supported.
 * Axis-aligned elements only (DSEM_ERR_UNSUPPORTED otherwise). */
int dsem_set_les(dsem_ctx *ctx, double cs, double numax);
/* The Smagorinsky model's shock and density sensors (DSEM's shockSensor and
 * rhoSensor inputs, input_lib.f90:163-164): nu_t is scaled by (1 - Ducros
 * sensor) and by the density-based sensor that the step's entropy viscosity
 * evaluates (staticSmag.f90:68-69, RHS.f90:264-275).  Without entropy
 * viscosity both sensors stay 0, as DSEM's zeroed arrays: the shock sensor
 * then leaves nu_t unchanged and the density sensor zeroes it. */
int dsem_set_les_sensors(dsem_ctx *ctx, int shock_sensor, int rho_sensor);
/* nu_t at Gauss points after the last evaluation (ldx layout, one field). */
int dsem_get_nut(dsem_ctx *ctx, double *nu, int ldx);

/* Checkpoint / resume of the device state (the solver-side part of DSEM's
 * write_restart / read_restart, Statistics/dongru/restart.f90:14-310, which
 * store d%Q and the Lobatto arrays d%Qlgg.. that entropy viscosity reads on
 * the next step).  The snapshot holds JQ, the last stage's gradients and the
 * diagnostics' previous kinetic energy, in the library's own versioned
 * layout; it loads only into a context built on the same mesh, and a run
 * resumed from it continues bit for bit. */
int dsem_state_size(const dsem_ctx *ctx, long long *nbytes);
int dsem_save_state(dsem_ctx *ctx, void *buf, long long nbytes);
int dsem_load_state(dsem_ctx *ctx, const void *buf, long long nbytes);

/* ---- Autotuning of the volume kernel's launch shape ----
 * No counterpart in DSEM (its element loops have no launch shape).  For each
 * element order of the context, times the launch shapes of the volume kernel
 * (threads per element, elements held per SM) on the context's own elements
 * and current state, `reps` launches each, and keeps the fastest for the
 * following steps.  Shapes exist for p = 4, 6 and 8 (other orders have one);
 * all give identical results.  choice[p-1] receives the chosen shape of order p
 * and ms[(p-1)*DSEM_VOL_VARIANTS + v] the mean time of shape v (-1: not timed);
 * either may be NULL.  Call it after dsem_upload_q.  dsem_set_vol_variant
 * sets a shape by hand. */
#define DSEM_MAX_ORDER 8
#define DSEM_VOL_VARIANTS 5
int dsem_autotune(dsem_ctx *ctx, int reps, int *choice, double *ms);
int dsem_set_vol_variant(dsem_ctx *ctx, int p, int variant);

/* ---- Boundary faces (mortars with id(2) = 0) ----
 * Sets the wall temperature of isothermal walls (MODULE physics twall) and,
 * for inflow and outflow faces, the external state and viscous flux that DSEM
 * keeps in mrtr%Q(:,:,:,2) and mrtr%fv(:,:,:,2) (set by initc / exactsol and
 * updated between steps by inflow_time_bc, BackstepProblem-stoch.f90:1275-1443,
 * 2077-2165).  Qext and fvext are [nmort][5][ldx][ldx] over all mortars of the
 * descriptor, point (i,j) of variable v of mortar k at i + ldx*(j + ldx*(v +
 * 5*k)); only boundary mortars are read.  Either may be NULL (fvext starts at
 * zero).  Call it before the first stage when the mesh has isothermal walls
 * (twall) or inflow/outflow faces (Qext); stepping fails otherwise.  It may be
 * called again between steps. */
int dsem_set_boundary(dsem_ctx *ctx, double twall, const double *Qext, const double *fvext, int ldx);

/* ---- One case sharded over several GPUs (one context per GPU) ----
 * The replacement for DSEM's MPI face exchange (send_q_to_mortars_mpi,
 * send_flux_to_mortars_mpi, add_flux_mpi: send_q.f90:771-895,
 * send_flux.f90:464-692, 1109-1206).  Each shard's descriptor holds its own
 * elements; a mortar whose other side is on another shard is "cut": that
 * side's element id is -(g+1), g (0-based) numbering the shard's ghost faces
 * 0..ncut-1.  A stage runs in three phases with two exchanges between them:
 *   phase 0: stage start; the local faces of the cut mortars (their face
 *            traces) are packed into `send`, block g for ghost g;
 *   exchange: the caller makes `ghost` block g the remote shard's `send`
 *            block of the same mortar (NCCL send/recv over NVLink, or any copy);
 *   phase 1: inviscid mortars (cut ones read the ghost traces), volume; the
 *            viscous face fluxes of the cut faces are packed into `send`;
 *   exchange again;
 *   phase 2: viscous mortars, update.
 * Both shards evaluate a cut mortar's points with the same operands, so a
 * sharded run reproduces the single-context run bit for bit.  Conforming cut
 * mortars of one element order; dsem_step / dsem_stage / dsem_rhs reject
 * sharded contexts.  dsem_diag_sums returns this shard's diagnostic sums
 * {sum u^2 w, v^2 w, w^2 w, |w|^2 J, J, jacob(1,1,1) of its element 1,
 * gradients valid}: the caller adds them over shards (an all-reduce) and
 * forms KE and eps as dsem_diag does. */
int dsem_shard_info(const dsem_ctx *ctx, int *nghost, int *doubles_per_face, double **send, double **ghost);
int dsem_shard_stage(dsem_ctx *ctx, double dt, int kk, int phase);
int dsem_diag_sums(dsem_ctx *ctx, double *sums);
/* Stream-ordered form of the same phases, for a caller that orders its
 * exchange on the context's stream (an NCCL send/recv issued on that stream
 * after phase 0 or 1 and before the next phase): dsem_shard_enqueue enqueues a
 * phase and returns without waiting; dsem_shard_finish waits for the stream
 * and reports a non-finite stage (DSEM_ERR_NONFINITE), once per step or
 * before the state is read; dsem_get_stream returns the context's CUDA stream
 * (a cudaStream_t).  No host round trip is needed between phases. */
int dsem_shard_enqueue(dsem_ctx *ctx, double dt, int kk, int phase);
int dsem_shard_finish(dsem_ctx *ctx);
int dsem_get_stream(const dsem_ctx *ctx, void **stream);

/* ---- DSEM restart files (write_restart / read_restart) ----
 * Replace write_restart / read_restart (src/Parabolic3D/stac3m/restart.f90:
 * 19-312, 319-929; called at 3DDriver_parfmdf.f90:516,622) for a context's
 * state: the file is DSEM's own Fortran unformatted sequential layout (one
 * record per WRITE, 4-byte lengths around each), so DSEM can restart from a
 * file the library wrote and the library from a file DSEM wrote.
 * dsem_keep_lobatto(ctx, 1): the last stage of every step also stores its
 *   three Lobatto arrays (d%Qlgg, d%Qglg, d%Qggl), which the file carries for
 *   the entropy viscosity of the next step (off by default; costs one extra
 *   kernel per step and [elements][3][5][(p+2)(p+1)^2] doubles of memory).
 * dsem_write_restart(ctx, template, out, max_materials, time): copies
 *   `template` -- a restart file DSEM wrote for the same mesh, e.g. by the
 *   serial zero-step run of its restart workflow -- record by record into
 *   `out`, with each element's Q and g_Q, and its Lobatto arrays when kept,
 *   taken from the device, and the time in the case record; every other
 *   record passes through.  max_materials is size.f90's (1 in DSEM's cases).
 * dsem_read_restart(ctx, path, max_materials, &time): uploads Q from the file;
 *   when its Lobatto arrays were computed (a file written after a step), the
 *   gradients the next step's entropy viscosity and Smagorinsky model read
 *   are rebuilt from them, so the run continues as if it had not stopped;
 *   zeroed arrays (DSEM's zero-step file) give a fresh start (mu_EV = 0 on
 *   the first step).  One-case, unsharded contexts; the padding nx of the
 *   file's (nx,nx,nx,5) arrays is read from the records. */
int dsem_keep_lobatto(dsem_ctx *ctx, int on);
int dsem_write_restart(dsem_ctx *ctx, const char *template_path, const char *out_path, int max_materials,
                       double time);
int dsem_read_restart(dsem_ctx *ctx, const char *path, int max_materials, double *time);

/* ---- Ensembles: ncase independent runs in one context ----
 * No DSEM counterpart (DSEM runs one case per job; each would call tstep,
 * tstep.f90:12, from its own time loop, 3DDriver_parfmdf.f90:466).  The
 * cases' elements share the launches: one launch per kernel type and element
 * order per stage for the whole ensemble, one CUDA graph per step, order
 * groups as parallel graph branches.  Each case keeps its own mesh (with its
 * own ldx), Reynolds number, time step, state and diagnostics; every case
 * gives bit-for-bit the result of its own single-case context.
 * meshes[ncase], phys[ncase]: all cases must share gamma, pr, mach, cmu,
 * mumax, shock and iord (DSEM_ERR_UNSUPPORTED otherwise); re may differ.
 * The descriptors' arrays are read only during the call.  Mortar ids are
 * per case (1-based within the case).  dsem_step / dsem_stage on an
 * ensemble use the same dt for every case; dsem_upload_q / dsem_download_q
 * / dsem_rhs see the cases' elements concatenated in case order. */
int dsem_create_batch(int ncase, const dsem_mesh_desc *meshes, const dsem_phys *phys, dsem_ctx **out);
int dsem_batch_size(const dsem_ctx *ctx); /* number of cases (1 for dsem_create) */
int dsem_upload_q_case(dsem_ctx *ctx, int icase, const double *JQ, int ldx);
int dsem_download_q_case(dsem_ctx *ctx, int icase, double *JQ, int ldx);
/* nsteps steps of every case, case k with time step dt[k] (tstep.f90:36-116). */
int dsem_step_batch(dsem_ctx *ctx, const double *dt, int nsteps);
/* dsem_diag per case: dt, ke, dkdt, eps are arrays of ncase (dsem_diag itself
 * rejects contexts with more than one case). */
int dsem_diag_batch(dsem_ctx *ctx, const double *dt, int first, double *ke, double *dkdt, double *eps);

/* ---- Discrete adjoint ----
 * No DSEM counterpart (DSEM has no adjoint solver).  Objective:
 *   J = sum over the last `window` of `nsteps` steps of eps_n * dt,
 * eps_n being the enstrophy dissipation dsem_diag reports after step n
 * (100 <|w|^2>/Re from the JQ values after the step and the gradients of its
 * last stage, energydissipation.f90:2-89).  Advances nsteps steps of size dt
 * from the current state (tstep.f90:36-116), then runs the exact discrete
 * adjoint of those steps backwards.  snapshots == 0 keeps every stage state
 * in device memory (nsteps * kord states); snapshots = s > 0 keeps s step
 * states and recomputes steps in binomial checkpointing order.  Outputs (each
 * may be NULL): J; dJ/d(JQ at the start) in the ldx layout of dsem_upload_q;
 * dJ/d(1/Re); the device milliseconds of the whole call.  The state is
 * restored on return.  Supported: one case, any element orders (p <= 8, with
 * the p-nonconforming mortars between them), axis-aligned elements, shock = 0, 1 or 3
 * (entropy viscosity, with or without the Ducros sensor) or static Smagorinsky LES without the
 * shock and density sensors (not both models at once; with snapshots > 0
 * each snapshot also keeps the gradients its step's viscosity reads),
 * boundary faces of every kind (walls, inflow, outflow; with them
 * DSEM_ADJ_SEGMENTS falls back to revolve), no sharding
 * (DSEM_ERR_UNSUPPORTED otherwise). */
int dsem_adjoint(dsem_ctx *ctx, double dt, int nsteps, int window, int snapshots, double *J, double *dJdQ0,
                 int ldx, double *dJdinvRe, double *ms);

/* How dsem_adjoint recomputes steps when snapshots = s > 0.
 * DSEM_ADJ_REVOLVE (the default): s step states, binomial checkpointing
 *   (Griewank's revolve order): the fewest recomputed steps for s stored states.
 * DSEM_ADJ_SEGMENTS: two levels.  The first sweep keeps the state at the start
 *   of each of ceil(nsteps / K) segments of K = ceil(nsteps / s) steps; the
 *   reverse sweep recomputes one segment at a time from its snapshot and keeps
 *   that segment's K * kord stage states and their face traces in device memory
 *   while it reverses the segment (the last segment is kept by the first sweep).
 *   Every step is recomputed at most once, for K * kord more stage states of
 *   device memory.  When those do not fit, the call falls back to revolve.
 * Both give the store-all gradient (snapshots == 0) bit for bit. */
#define DSEM_ADJ_REVOLVE 0
#define DSEM_ADJ_SEGMENTS 1
int dsem_set_adjoint_scheme(dsem_ctx *ctx, int scheme);

/* Size of the static device array that holds the working buffers of
 * dsem_rhs_noalloc: 2^20 doubles (8 MiB) on every GPU that loads the library. */
#define DSEM_NOALLOC_SCRATCH_DOUBLES (1 << 20)

/* No counterpart in the reference (DSEM's Fortran allocates all its arrays at
 * start-up and has no GPU path).  The right-hand side of dsem_rhs for callers
 * that cannot allocate device memory -- applications whose GPU memory is owned
 * by their own pool allocator or fixed at start-up, where a cudaMalloc inside a
 * library fails or breaks their budget.  It allocates nothing: inputs and output
 * are the caller's device arrays, and the working buffers live in one static
 * device array of DSEM_NOALLOC_SCRATCH_DOUBLES doubles.
 *   Limits: one order p (1..8) for every element, fully periodic conforming
 *   mesh, axis-aligned (diagonal) metrics, and
 *   nel*(90*(p+1)^2 + 5*(p+1)^3) + 1 <= DSEM_NOALLOC_SCRATCH_DOUBLES
 *   (95 elements at p = 8, 364 at p = 4); larger meshes are rejected with
 *   DSEM_ERR_INVALID_ARG and a message from dsem_last_error(NULL).
 *   Device arrays (G = p+1, L = p+2, element-major, x fastest):
 *     mortar      [nmort][DSEM_MORTAR_INTS]  same rows as dsem_mesh_desc.mortar
 *     n_hat, norm [nmort][G*G][3], [nmort][G*G]  (mortar point i + G*j)
 *     JQ, Qt      [nel][5][G^3]   (Qt is the output, the rest are read)
 *     jac         [nel][G^3]      d%jacob
 *     gmetg_diag  [nel][3][G^3]   gmetg(d,d) at the Gauss points
 *     gmet_diag   [nel][3][L*G^2] gmet(d,d) on staggered grid d
 *   The first call on a device does a one-time set-up with that device current
 *   (scratch address, operator tables).  No call may be made while `stream` is
 *   being captured into a CUDA graph: each call clears the scratch, reads an
 *   error flag back and waits for the stream, and returns DSEM_ERR_INVALID_ARG
 *   on a capturing stream.  Mortar rows that are not conforming mortars of
 *   order p (len/lenmortar != p+1 or a conforming flag of 0) are refused with
 *   DSEM_ERR_UNSUPPORTED; rows with ids, faces or orientations out of range
 *   with DSEM_ERR_INVALID_ARG.
 *   Every call shares the scratch array and leaves its contents behind: calls
 *   whose work overlaps on the GPU race on it.  The call runs on `stream`
 *   (cudaStream_t, NULL = default stream) and waits for it before returning. */
int dsem_rhs_noalloc(int nel, int p, int nmort, const int *mortar, const double *n_hat, const double *norm,
                     const double *JQ, const double *jac, const double *gmetg_diag, const double *gmet_diag,
                     double gamma, double re, double pr, double mach, double *Qt, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* DSEM_GPU_H */
