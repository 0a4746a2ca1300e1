/*
 * dsem_oracle.h -- C API of the CPU oracle for the DSEM hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker: a CPU restatement
 * of DSEM's Fortran right-hand side, low-storage Runge-Kutta stage, entropy
 * viscosity and diagnostics, written from the reference sources (each
 * function in dsem_oracle.cpp cites the file:line it follows).  Only the
 * tests, the smoke check and the CPU-baseline leg of the benchmark may load
 * it.  The product (dsem_b200) never links, loads or calls it.
 *
 * Parity is unpinned against DSEM itself: the reference ships no golden
 * vectors and its Fortran toolchain (gfortran, MPI) is absent here, so the
 * restatement is pinned by known-answer tests derived from the mathematics
 * (operator exactness, freestream preservation, conservation, Roe
 * consistency, analytic Taylor-Green invariants).
 *
 * Array layouts follow the C-ABI of include/dsem_gpu.h (Fortran column-major
 * blocks with a caller-chosen padding extent ldx).
 */
#ifndef DSEM_ORACLE_H
#define DSEM_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_case orc_case;

/* Periodic box of nex*ney*nez straight hex8 elements on [0,lx]x[0,ly]x[0,lz].
 * Element numbering follows the shipped TGV mesh: y fastest, then x, then z.
 * orders[e] = polynomial order p of element e (ncg = p+1, nc = p+2).
 * rot[e] (may be NULL) = one of 24 rigid rotations of the element's local
 * axes (0 = identity); only interior elements may be rotated.
 * Mirrors read_mesh + generate_mortars + set_geometry + user_setup. */
orc_case *orc_build_box(int nex, int ney, int nez, double lx, double ly, double lz,
                        const int *orders, const int *rot);

/* Case from a mesh descriptor in the C-ABI layout (see include/dsem_gpu.h). */
orc_case *orc_from_desc(int ngrid, int nmort, int ldx, const int *ncg,
                        const double *jacob, const double *gmetg, const double *gmet,
                        const int *mortar, const double *n_hat, const double *norm);

void orc_free(orc_case *c);
void orc_set_phys(orc_case *c, double gamma, double re, double pr, double mach,
                  double cmu, double mumax, int shock, int iord);
int orc_nel(const orc_case *c);
int orc_nmort(const orc_case *c);
int orc_ncg(const orc_case *c, int e);

/* Export the descriptor arrays (caller allocates; ldx >= max ncg+1).
 * xg: [ngrid][ldx^3][3] physical Gauss point coordinates. */
void orc_export_desc(const orc_case *c, int ldx, int *ncg, double *jacob, double *gmetg,
                     double *gmet, int *mortar, double *n_hat, double *norm, double *xg);

/* Operator matrices of one order: dmx [G][L] (row k = Gauss point), bx [L][G]. */
void orc_operators(int p, double *dmx, double *bx);
/* Mortar projection matrices (compute_pmat): prolong [nout][nin], restrict [nin][nout]. */
void orc_projection(int nin, int nout, double *prolong, double *restrict_);
/* KE quadrature weights bmatu1b [G][G][G] (Fortran (i,j,l), i fastest). */
void orc_ke_weights(int G, double *w);

/* Taylor-Green initial condition (initc/exactsol), stored as J*Q. */
void orc_init_tgv(orc_case *c, double twall, double v0);
void orc_set_q(orc_case *c, const double *JQ, int ldx);
void orc_get_q(const orc_case *c, double *JQ, int ldx);
int orc_get_lobatto(const orc_case *c, double *out, int ldx);
/* Inviscid time step (dtcalc), minimum over elements, before the CFL factor. */
double orc_dtcalc(const orc_case *c);

/* One evaluation of Fluxes at time tk followed by Qt (no update). */
void orc_rhs(orc_case *c, double tk, double *Qt, int ldx);
/* One Runge-Kutta stage kk (1-based): EV and g_Q zeroing at kk==1.
 * Qt (may be NULL) receives the stage right-hand side. Returns 0, or -3 if
 * resid is not finite. */
int orc_stage(orc_case *c, double time, double dt, int kk, double *Qt, int ldx);
/* nsteps full time steps (tstep), time advanced by dt each step. */
int orc_step(orc_case *c, double time, double dt, int nsteps);
/* do_user_stuff KE (turbk), -dKE/dt with prestep state, and energydissipation. */
void orc_diag(orc_case *c, double dt, int first, double *turbk, double *dissp, double *enst);
/* Entropy-viscosity coefficient at Gauss points after the last EV evaluation. */
void orc_get_muhg(const orc_case *c, double *mu, int ldx);
int orc_set_threads(int n);
int orc_kord(const orc_case *c);
/* Pointwise physics for unit tests: Roe flux (PhysLib.f90:231-320), Euler and
 * viscous fluxes (PhysLib.f90:17-124, 419-583). */
void orc_riemann(const double *n_hat, double ds, const double *Ql, const double *Qr, double gamma, double *flux);
void orc_euler(const double *Q, double gamma, double *f, double *g, double *h);
void orc_vis(const double *Q, const double *Qx, const double *Qy, const double *Qz, double amu, double gamma,
             double pr, double mach, double *f, double *g, double *h);
void orc_rk(const orc_case *c, double *ark, double *brk, double *crk);
/* Static Smagorinsky LES (staticSmag.f90) with coefficient cs (0: off) and
 * clip numax; evaluated at the start of each step like the entropy viscosity.
 * orc_get_nut: its Gauss-point viscosity after the last evaluation. */
void orc_set_les(orc_case *c, double cs, double numax);
void orc_set_les_sensors(orc_case *c, int shock_sensor, int rho_sensor);
/* boundary faces: d%bcond per element face ([ngrid][6]: 1 walladiab, 2 wallisoth,
 * 3 inflow, 4 outflow), then twall and the external mortar states
 * ([nmort][5][ldx][ldx], i fastest; null without inflow/outflow faces) */
int orc_set_bcond(orc_case *c, const int *bcond);
void orc_set_boundary(orc_case *c, double twall, const double *Qx, const double *fvx, int ldx);
void orc_get_nut(const orc_case *c, double *nu, int ldx);
/* Objective of the adjoint, J = sum over the last `window` of `nsteps` steps of
 * dt * enst (orc_diag's enstrophy dissipation after each step), evaluated from
 * the current state + i*hstep*dq in complex arithmetic: *J = Re J and
 * *dJ = Im J / hstep (the directional derivative along dq).  The case is not
 * modified. */
void orc_objective_cs(const orc_case *c, double dt, int nsteps, int window, const double *dq, double hstep, int ldx,
                      double *J, double *dJ);

#ifdef __cplusplus
}
#endif
#endif
