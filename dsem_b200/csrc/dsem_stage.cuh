// dsem_stage.cuh -- the per-stage kernels.
//
//  k_trace   : physical Q traces on the six faces          (Int_fluxes face slots)
//  k_face_inv: Roe flux + averaged state per mortar point  (interface_flux, V_Avg_Soln,
//                                                           send_flux_to_faces, send_q_to_faces)
//  k_vol     : Lobatto arrays, Gauss gradients, viscous + inviscid fluxes on the three
//              staggered grids, interior flux divergence   (Int_fluxes, Vis_Fluxes,
//                                                           Gauss_Deriv, update_interior)
//  k_face_vis: BR1 average of the viscous normal flux      (send_flux_to_mortars,
//                                                           mortar_vis_flux, send_flux_to_faces_add)
//  k_update  : face terms of the divergence, 2N-storage update, next-stage traces
//  k_ev      : entropy-viscosity coefficient at Gauss points (RHS_ent_trans, Entropy_Viscosity)
#pragma once
#include "dsem_kernels.cuh"

#ifdef DSEM_PHASE_TIMING
// development probe: cycles per phase of the volume kernel, summed over blocks
__device__ unsigned long long g_phase_cycles[32];
#define PHASE_MARK(i)                                                  \
  do {                                                                 \
    if (threadIdx.x == 0) {                                            \
      long long now_ = clock64();                                      \
      atomicAdd(&g_phase_cycles[i], (unsigned long long)(now_ - t_ph_)); \
      t_ph_ = now_;                                                    \
    }                                                                  \
  } while (0)
#else
#define PHASE_MARK(i) \
  do {                \
  } while (0)
#endif

#ifndef DSEM_VOL_THREADS_P8
#define DSEM_VOL_THREADS_P8 448  // threads per volume CTA for p >= 7 (fastest of 384/448/512 at p = 8)
#endif

namespace dsem {

// ------------------------------------------------------------------ traces
template <int G, int HI> __device__ __forceinline__ double trace_of(const double *x, int xs) {
  constexpr int n = HI ? G : 0;  // Lobatto end point (L-1 = G)
  double acc = Op<G>::B(n, 0) * x[0];
#pragma unroll
  for (int j = 1; j < G; ++j) acc = __fma_rn(Op<G>::B(n, j), x[j * xs], acc);
  return acc;
}

// all six face traces of the 5 fields in q (Gauss layout, smem) -> QF slots
template <int G> __device__ __forceinline__ void write_traces(const double *q, double *QF, int tid, int nt) {
  constexpr int G2 = G * G, NG = G * G * G;
  for (int t = tid; t < 30 * G2; t += nt) {
    const int f = t / (5 * G2);  // 0..5 -> faces 1..6
    const int r = t - f * 5 * G2;
    const int v = r / G2, ln = r - v * G2;
    const int a = ln % G, b = ln / G;
    const int face = f + 1;
    const int d = (face == 4 || face == 6) ? 0 : ((face == 1 || face == 2) ? 1 : 2);
    const double *x = q + v * NG;
    double val;
    if (d == 0) {
      x += gbase<G>(0, a, b);
      val = (face == 4) ? trace_of<G, 1>(x, 1) : trace_of<G, 0>(x, 1);
    } else if (d == 1) {
      x += gbase<G>(1, a, b);
      val = (face == 2) ? trace_of<G, 1>(x, G) : trace_of<G, 0>(x, G);
    } else {
      x += gbase<G>(2, a, b);
      val = (face == 5) ? trace_of<G, 1>(x, G2) : trace_of<G, 0>(x, G2);
    }
    QF[t] = val;
  }
}

struct TraceArgs {
  const double *JQ;
  long long sq;
  const double *jac;
  double *QF;
};

template <int G> __global__ void __launch_bounds__(256) k_trace(TraceArgs A) {
  constexpr int G2 = G * G, NG = G * G * G;
  extern __shared__ double sm[];
  const int k = blockIdx.x, tid = threadIdx.x, nt = blockDim.x;
  const double *JQ = A.JQ + (long long)k * A.sq;
  const double *jac = A.jac + (long long)k * NG;
  for (int i = tid; i < 5 * NG; i += nt) sm[i] = JQ[i] * jac[i % NG];
  __syncthreads();
  write_traces<G>(sm, A.QF + (long long)k * 30 * G2, tid, nt);
}

// --------------------------------------------------------------- face kernels
// Conforming mortar: master slot, slave slot (offsets in the face buffers),
// geometry index, flags = orient | (sign<0)<<3 | (nsign<0)<<4 | (master face low)<<5.
struct MortarC {
  long long ms, ss;
  int geo, flags;
};

// mortar index (i,j) -> slave face index (rotate_to_mortar inverse, mortar_operations.f90:461-605)
template <int G> __device__ __forceinline__ void slave_index(int orient, int i, int j, int &si, int &sj) {
  switch (orient) {
    case 3: si = i; sj = G - 1 - j; break;          // F1B2
    case 2: si = G - 1 - i; sj = G - 1 - j; break;  // B1B2
    case 1: si = G - 1 - i; sj = j; break;          // B1F2
    case 4: si = j; sj = i; break;                  // F2F1
    case 5: si = j; sj = G - 1 - i; break;          // B2F1
    case 6: si = G - 1 - j; sj = G - 1 - i; break;  // B2B1
    case 7: si = G - 1 - j; sj = i; break;          // F2B1
    default: si = i; sj = j; break;
  }
}

// Roe flux and averaged state at one mortar point, from the raw traces in QFin
// to the averages in QF (QFin == QF: in place; each point is read and written by
// its own thread only).
template <int G>
__device__ __forceinline__ void face_inv_point(const MortarC &M, int pt, const double *QFin, double *QF,
                                               double *__restrict__ FF, const double *__restrict__ nh,
                                               const double *__restrict__ nrm, double gamma) {
  constexpr int G2 = G * G;
  const int i = pt % G, j = pt / G;
  int si, sj;
  slave_index<G>(M.flags & 7, i, j, si, sj);
  const int sp = si + G * sj;
  double Q1[NV], Q2[NV], f[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    Q1[v] = QFin[M.ms + v * G2 + pt];
    Q2[v] = QFin[M.ss + v * G2 + sp];
  }
  const long long gp = (long long)M.geo * G2 + pt;
  const double n3[3] = {nh[gp * 3], nh[gp * 3 + 1], nh[gp * 3 + 2]};
  const bool low = (M.flags >> 5) & 1;
  riemann(n3, nrm[gp], low ? Q2 : Q1, low ? Q1 : Q2, gamma, f);
  const double sgn = ((M.flags >> 3) & 1) ? -1.0 : 1.0;
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    const double avg = (Q1[v] + Q2[v]) * 0.5;
    FF[M.ms + v * G2 + pt] = f[v];
    FF[M.ss + v * G2 + sp] = sgn * f[v];
    QF[M.ms + v * G2 + pt] = avg;
    QF[M.ss + v * G2 + sp] = avg;
  }
}

template <int G>
__global__ void __launch_bounds__(128) k_face_inv(const MortarC *__restrict__ mc, int nm, double *QF,
                                                   double *__restrict__ FF, const double *__restrict__ nh,
                                                   const double *__restrict__ nrm, double gamma) {
  constexpr int G2 = G * G;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)nm * G2) return;
  const int m = (int)(t / G2), pt = (int)(t - (long long)m * G2);
  face_inv_point<G>(mc[m], pt, QF, QF, FF, nh, nrm, gamma);
}

// The same with the raw traces kept elsewhere (QFR, left unchanged).
template <int G>
__global__ void __launch_bounds__(128) k_face_inv_from(const MortarC *__restrict__ mc, int nm,
                                                        const double *__restrict__ QFR, double *__restrict__ QF,
                                                        double *__restrict__ FF, const double *__restrict__ nh,
                                                        const double *__restrict__ nrm, double gamma) {
  constexpr int G2 = G * G;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)nm * G2) return;
  const int m = (int)(t / G2), pt = (int)(t - (long long)m * G2);
  face_inv_point<G>(mc[m], pt, QFR, QF, FF, nh, nrm, gamma);
}

template <int G>
__global__ void __launch_bounds__(128) k_face_vis(const MortarC *__restrict__ mc, int nm, double *__restrict__ VF,
                                                   const double *__restrict__ nrm) {
  constexpr int G2 = G * G;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)nm * G2) return;
  const int m = (int)(t / G2), pt = (int)(t - (long long)m * G2);
  const MortarC M = mc[m];
  const int i = pt % G, j = pt / G;
  int si, sj;
  slave_index<G>(M.flags & 7, i, j, si, sj);
  const int sp = si + G * sj;
  const long long g0 = (long long)M.geo * G2;
  const double nm_m = nrm[g0 + pt], nm_s = nrm[g0 + sp];
  const double rm = 1.0 / nm_m, rs = 1.0 / nm_s;
  const bool neg_n = (M.flags >> 4) & 1, neg_s = (M.flags >> 3) & 1;
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    const double fv1 = ddiv(VF[M.ms + v * G2 + pt], nm_m, rm);
    const double fv2 = ddiv(VF[M.ss + v * G2 + sp], nm_s, rs);
    const double Qs = neg_n ? -fv2 : fv2;
    const double qb = 0.5 * (fv1 + Qs) * nm_m;
    VF[M.ms + v * G2 + pt] = qb;
    VF[M.ss + v * G2 + sp] = neg_s ? -qb : qb;
  }
}

// --------------------------------------------------------- cut mortars
// A conforming mortar whose other side lives on another shard (another GPU):
// the local face slot ls, the remote face's data (its own face layout) at ghost
// offset go of the ghost buffer, flags as MortarC plus (local side is master)<<6.
// Both shards evaluate the same point with the same operands and each writes
// only its own side, so the result equals the unsharded kernels' bit for bit.
struct MortarCut {
  long long ls, go;
  int geo, flags;
};

template <int G>
__global__ void __launch_bounds__(128) k_face_inv_cut(const MortarCut *__restrict__ mc, int nm, double *__restrict__ QF,
                                                       double *__restrict__ FF, const double *__restrict__ ghost,
                                                       const double *__restrict__ nh, const double *__restrict__ nrm,
                                                       double gamma) {
  constexpr int G2 = G * G;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)nm * G2) return;
  const int m = (int)(t / G2), pt = (int)(t - (long long)m * G2);
  const MortarCut M = mc[m];
  int si, sj;
  slave_index<G>(M.flags & 7, pt % G, pt / G, si, sj);
  const int sp = si + G * sj;
  const bool lm = (M.flags >> 6) & 1;
  double Q1[NV], Q2[NV], f[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    Q1[v] = lm ? QF[M.ls + v * G2 + pt] : ghost[M.go + v * G2 + pt];
    Q2[v] = lm ? ghost[M.go + v * G2 + sp] : QF[M.ls + v * G2 + sp];
  }
  const long long gp = (long long)M.geo * G2 + pt;
  const double n3[3] = {nh[gp * 3], nh[gp * 3 + 1], nh[gp * 3 + 2]};
  const bool low = (M.flags >> 5) & 1;
  riemann(n3, nrm[gp], low ? Q2 : Q1, low ? Q1 : Q2, gamma, f);
  const double sgn = ((M.flags >> 3) & 1) ? -1.0 : 1.0;
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    const double avg = (Q1[v] + Q2[v]) * 0.5;
    if (lm) {
      FF[M.ls + v * G2 + pt] = f[v];
      QF[M.ls + v * G2 + pt] = avg;
    } else {
      FF[M.ls + v * G2 + sp] = sgn * f[v];
      QF[M.ls + v * G2 + sp] = avg;
    }
  }
}

template <int G>
__global__ void __launch_bounds__(128) k_face_vis_cut(const MortarCut *__restrict__ mc, int nm, double *__restrict__ VF,
                                                       const double *__restrict__ ghost, const double *__restrict__ nrm) {
  constexpr int G2 = G * G;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)nm * G2) return;
  const int m = (int)(t / G2), pt = (int)(t - (long long)m * G2);
  const MortarCut M = mc[m];
  int si, sj;
  slave_index<G>(M.flags & 7, pt % G, pt / G, si, sj);
  const int sp = si + G * sj;
  const bool lm = (M.flags >> 6) & 1;
  const long long g0 = (long long)M.geo * G2;
  const double nm_m = nrm[g0 + pt], nm_s = nrm[g0 + sp];
  const double rm = 1.0 / nm_m, rs = 1.0 / nm_s;
  const bool neg_n = (M.flags >> 4) & 1, neg_s = (M.flags >> 3) & 1;
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    const double vm = lm ? VF[M.ls + v * G2 + pt] : ghost[M.go + v * G2 + pt];
    const double vs = lm ? ghost[M.go + v * G2 + sp] : VF[M.ls + v * G2 + sp];
    const double fv1 = ddiv(vm, nm_m, rm);
    const double fv2 = ddiv(vs, nm_s, rs);
    const double Qs = neg_n ? -fv2 : fv2;
    const double qb = 0.5 * (fv1 + Qs) * nm_m;
    if (lm)
      VF[M.ls + v * G2 + pt] = qb;
    else
      VF[M.ls + v * G2 + sp] = neg_s ? -qb : qb;
  }
}

// send[g] = the local face slot src[g] (5 fields of G^2 points) of field array F
static __global__ void k_pack_cut(const long long *__restrict__ src, int nghost, int nper, const double *__restrict__ F,
                           double *__restrict__ send) {
  const long long n = (long long)nghost * nper;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const long long g = i / nper, r = i - g * nper;
    send[i] = F[src[g] + r];
  }
}

// ------------------------------------------------------- boundary faces
// Mortars without a neighbour (id(2) = 0), conforming with orient 0: the master
// face only.  boundary_flux, DirichletBC and Vis_Neumann of the problem file
// (caseFiles/tgv/BackstepProblem-stoch.f90:1602-1729) dispatch on the master
// face's d%bcond to the routines of NS/BCs/stac3m restated below.
enum { BC_WALLADIAB = 1, BC_WALLISOTH = 2, BC_INFLOW = 3, BC_OUTFLOW = 4 };
struct MortarB {
  long long ms;  // master face slot
  int geo;       // index in the order's boundary list (geometry, external state)
  int flags;     // condition (bits 0-2) | master face 1, 3 or 6 (bit 3) | nsign < 0 (bit 4)
};
struct BndPhys {
  double gamma, twall, r_cv;  // r_cv = 1 / (mach^2 gamma (gamma-1)), correctly rounded
  double cv;                  // mach^2 gamma (gamma-1)
};

// External state of a wall: density and energy kept, normal momentum reversed
// (wallbc_inv.f90:32-50, wallbc_isoth2.f90:31-54).
__device__ __forceinline__ void wall_mirror(const double *nh, const double *Q1, double *Q2) {
  const double qnorm = nh[0] * Q1[1] + nh[1] * Q1[2] + nh[2] * Q1[3];
  const double tx = Q1[1] - qnorm * nh[0], ty = Q1[2] - qnorm * nh[1], tz = Q1[3] - qnorm * nh[2];
  Q2[0] = Q1[0];
  Q2[1] = tx - qnorm * nh[0];
  Q2[2] = ty - qnorm * nh[1];
  Q2[3] = tz - qnorm * nh[2];
  Q2[4] = Q1[4];
}

// osher (PhysLib.f90:698-790): the state between the normal Riemann
// invariants of Ql and Qr, then its Euler flux (fflux/gflux/hflux :17-124)
// along n scaled by ds.
static __device__ __noinline__ void osher_flux(const double *nh, double ds, const double *Ql, const double *Qr, double gamma,
                                        double *flux) {
  const double en1 = nh[0], en2 = nh[1], en3 = nh[2];
  const double rho = Ql[0], rhou = Ql[1], rhov = Ql[2], rhow = Ql[3], rhoe = Ql[4];
  const double rhon = Qr[0], rhoun = Qr[1], rhovn = Qr[2], rhown = Qr[3], rhoen = Qr[4];
  const double qdotn = (en1 * rhou + en2 * rhov + en3 * rhow) / rho;
  const double qdotnn = (en1 * rhoun + en2 * rhovn + en3 * rhown) / rhon;
  const double p = (gamma - 1.0) * (rhoe - 0.5 / rho * (rhou * rhou + rhov * rhov + rhow * rhow));
  const double a = sqrt(gamma * p / rho);
  double pn = (gamma - 1.0) * (rhoen - 0.5 / rhon * (rhoun * rhoun + rhovn * rhovn + rhown * rhown));
  const double an = sqrt(gamma * pn / rhon);
  const double q_tanx = rhoun / rhon - qdotnn * en1;
  const double q_tany = rhovn / rhon - qdotnn * en2;
  const double q_tanz = rhown / rhon - qdotnn * en3;
  const double z = (gamma - 1.0) / (2.0 * gamma);
  double Ha = -qdotnn / an + 2.0 / (gamma - 1.0);
  Ha = Ha / (qdotn / a + 2.0 / (gamma - 1.0));
  pn = p / pow(Ha, 1.0 / z);
  double pstar = a + an - (qdotnn - qdotn) * (gamma - 1.0) / 2.0;
  pstar = pstar / (a / pow(p, z) + an / pow(pn, z));
  pstar = pow(pstar, 1.0 / z);
  double ustar = Ha * qdotn / a + qdotnn / an + 2.0 * (Ha - 1.0) / (gamma - 1.0);
  ustar = ustar / (Ha / a + 1.0 / an);
  const double rs = pstar * gamma / (an * an);
  const double u = q_tanx + en1 * ustar, v = q_tany + en2 * ustar, w = q_tanz + en3 * ustar;
  const double Q0 = rs, Q1 = rs * u, Q2 = rs * v, Q3 = rs * w;
  const double Q4 = pstar / (gamma - 1.0) + 0.5 * rs * (u * u + v * v + w * w);
  // fflux / gflux / hflux of Q
  const double uu = Q1 / Q0, vv = Q2 / Q0, ww = Q3 / Q0;
  const double pp = (gamma - 1.0) * (Q4 - 0.5 * Q0 * (uu * uu + vv * vv + ww * ww));
  const double f[NV] = {Q1, pp + Q1 * uu, Q1 * vv, Q1 * ww, uu * (Q4 + pp)};
  const double g[NV] = {Q2, Q1 * vv, pp + Q2 * vv, Q3 * vv, vv * (Q4 + pp)};
  const double h[NV] = {Q3, Q1 * ww, Q2 * ww, pp + Q3 * ww, ww * (Q4 + pp)};
#pragma unroll
  for (int k = 0; k < NV; ++k) flux[k] = ds * (en1 * f[k] + en2 * g[k] + en3 * h[k]);
}

// riemann_solution (PhysLib.f90:326-412): the interface state from the normal
// Riemann invariants (Dirichlet values of inflow and outflow faces).
static __device__ __noinline__ void riemann_state(const double *nh, const double *Ql, const double *Qr, double gamma,
                                           double *Q) {
  const double en1 = nh[0], en2 = nh[1], en3 = nh[2];
  const double rho = Ql[0], rhou = Ql[1], rhov = Ql[2], rhow = Ql[3], rhoe = Ql[4];
  const double rhon = Qr[0], rhoun = Qr[1], rhovn = Qr[2], rhown = Qr[3], rhoen = Qr[4];
  const double qdotn = (en1 * rhou + en2 * rhov + en3 * rhow) / rho;
  const double qdotnn = (en1 * rhoun + en2 * rhovn + en3 * rhown) / rhon;
  const double p = (gamma - 1.0) * (rhoe - 0.5 / rho * (rhou * rhou + rhov * rhov + rhow * rhow));
  const double a = sqrt(gamma * p / rho);
  const double pn = (gamma - 1.0) * (rhoen - 0.5 / rhon * (rhoun * rhoun + rhovn * rhovn + rhown * rhown));
  const double an = sqrt(gamma * pn / rhon);
  const double e0 = 0.5 * (qdotn + qdotnn);
  const double eplus = e0 + 0.5 * (a + an);
  const double eminus = e0 - 0.5 * (a + an);
  double etos, q_tanx, q_tany, q_tanz;
  if (e0 > 0.0) {
    etos = p / pow(rho, gamma);
    q_tanx = rhou / rho - qdotn * en1;
    q_tany = rhov / rho - qdotn * en2;
    q_tanz = rhow / rho - qdotn * en3;
  } else {
    etos = pn / pow(rhon, gamma);
    q_tanx = rhoun / rhon - qdotnn * en1;
    q_tany = rhovn / rhon - qdotnn * en2;
    q_tanz = rhown / rhon - qdotnn * en3;
  }
  const double rplus = eplus >= 0.0 ? qdotn + 2.0 / (gamma - 1.0) * a : qdotnn + 2.0 / (gamma - 1.0) * an;
  const double rminus = eminus >= 0.0 ? qdotn - 2.0 / (gamma - 1.0) * a : qdotnn - 2.0 / (gamma - 1.0) * an;
  const double qn = 0.5 * (rplus + rminus);
  const double as = 0.25 * (gamma - 1.0) * (rplus - rminus);
  const double rs = pow(as * as / (gamma * etos), 1.0 / (gamma - 1.0));
  const double ps = pow(rs, gamma) * etos;
  const double u = q_tanx + en1 * qn, v = q_tany + en2 * qn, w = q_tanz + en3 * qn;
  Q[0] = rs;
  Q[1] = rs * u;
  Q[2] = rs * v;
  Q[3] = rs * w;
  Q[4] = ps / (gamma - 1.0) + 0.5 * rs * (u * u + v * v + w * w);
}

// Inviscid boundary faces (fluxesH_newa.f90:116-139): boundary_flux, then
// DirichletBC into the face's Q trace.  One thread per mortar point.
//  walladiab: Roe flux against the mirror state; Q trace (rho, 0, 0, 0, rhoE)
//             (wallbc_Inv; set_adiabatic_wall, ViscousBC_slide.f90:111-175)
//  wallisoth: the mirror state at the wall temperature, osher flux (normal
//             reversed on faces 1, 3, 6); Q trace (rho, 0, 0, 0, rho twall/cv)
//             (wallbc_isoth2.f90; set_isothermal_wall, ViscousBC_slide.f90:356-420)
//  inflow, outflow: Roe flux against the external state; Q trace from
//             riemann_solution (inflow_specAll / outflow_specAll; boundary_values
//             ViscousBC_slide.f90:9-102)
template <int G>
__global__ void __launch_bounds__(128) k_face_bnd_inv(const MortarB *__restrict__ mb, int nm, double *__restrict__ QF,
                                                       double *__restrict__ FF, const double *__restrict__ nh,
                                                       const double *__restrict__ nrm, const double *__restrict__ qext,
                                                       BndPhys P) {
  constexpr int G2 = G * G;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)nm * G2) return;
  const int m = (int)(t / G2), pt = (int)(t - (long long)m * G2);
  const MortarB M = mb[m];
  const int bc = M.flags & 7;
  const bool low = (M.flags >> 3) & 1;
  double Q1[NV], Q2[NV], f[NV], qb[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) Q1[v] = QF[M.ms + v * G2 + pt];
  const long long gp = (long long)M.geo * G2 + pt;
  const double n3[3] = {nh[gp * 3], nh[gp * 3 + 1], nh[gp * 3 + 2]};
  const double ds = nrm[gp];
  if (bc == BC_WALLADIAB || bc == BC_WALLISOTH) {
    wall_mirror(n3, Q1, Q2);
    if (bc == BC_WALLADIAB) {
      riemann(n3, ds, low ? Q2 : Q1, low ? Q1 : Q2, P.gamma, f);
      qb[4] = Q1[4];
    } else {
      const double rho = Q2[0];
      const double u = Q2[1] / rho, v = Q2[2] / rho, w = Q2[3] / rho;
      Q2[4] = ddiv(rho * P.twall, P.cv, P.r_cv) + 0.5 * rho * (u * u + v * v + w * w);
      if (low) {
        const double mn[3] = {-n3[0], -n3[1], -n3[2]};
        osher_flux(mn, -ds, Q1, Q2, P.gamma, f);
      } else {
        osher_flux(n3, ds, Q1, Q2, P.gamma, f);
      }
      qb[4] = ddiv(Q1[0] * P.twall, P.cv, P.r_cv);
    }
    qb[0] = Q1[0];
    qb[1] = qb[2] = qb[3] = 0.0;
  } else {
#pragma unroll
    for (int v = 0; v < NV; ++v) Q2[v] = qext[(long long)M.geo * NV * G2 + v * G2 + pt];
    riemann(n3, ds, low ? Q2 : Q1, low ? Q1 : Q2, P.gamma, f);
    riemann_state(n3, low ? Q2 : Q1, low ? Q1 : Q2, P.gamma, qb);
  }
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    FF[M.ms + v * G2 + pt] = f[v];
    QF[M.ms + v * G2 + pt] = qb[v];
  }
}

// Viscous boundary faces: Vis_Neumann (Vis_Fluxes_new.f90:337-343).  Walls
// keep the face's own viscous flux, with a zero energy flux on adiabatic walls
// (wall_vis_flux, ViscousBC_slide.f90:279-348); inflow and outflow average it
// with the external one (boundary_vis_flux, :183-225).
template <int G>
__global__ void __launch_bounds__(128) k_face_bnd_vis(const MortarB *__restrict__ mb, int nm, double *__restrict__ VF,
                                                       const double *__restrict__ nrm,
                                                       const double *__restrict__ fvext) {
  constexpr int G2 = G * G;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)nm * G2) return;
  const int m = (int)(t / G2), pt = (int)(t - (long long)m * G2);
  const MortarB M = mb[m];
  const int bc = M.flags & 7;
  const bool neg_n = (M.flags >> 4) & 1;
  const long long gp = (long long)M.geo * G2 + pt;
  const double nm_m = nrm[gp], rm = 1.0 / nm_m;
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    const double fv1 = ddiv(VF[M.ms + v * G2 + pt], nm_m, rm);
    double qb;
    if (bc == BC_WALLADIAB || bc == BC_WALLISOTH) {
      qb = (v == 4 && bc == BC_WALLADIAB) ? 0.0 : fv1 * nm_m;
    } else {
      const double fx = fvext[(long long)M.geo * NV * G2 + v * G2 + pt];
      const double Qs = neg_n ? -fx : fx;
      qb = 0.5 * (fv1 + Qs) * nm_m;
    }
    VF[M.ms + v * G2 + pt] = qb;
  }
}

// ------------------------------------------------------- nonconforming faces
// One CTA per p-nonconforming mortar (lenmortar > len on at least one side).
// Mirrors interface_flux / map_to_mortar_space / map_to_face_space /
// rotate_to_mortar / rotate_flux_to_face (mortar_operations.f90:151-758) with
// the consistent prolong -> flux/average -> restrict sequence.  Arrays are
// [var][j*NMX + i] in shared memory.
constexpr int NMX = GMAX + 1;  // mortar extents never exceed GMAX
struct MortarNC {
  long long ms, ss;          // face slot offsets (master, slave)
  int gm, gs;                // Gauss points per direction on each side
  int lm1, lm2;              // lenmortar
  int orient, sign, nsign, low;
  int conf[4];               // conforming (dir1,side1) (dir2,side1) (dir1,side2) (dir2,side2)
  int geo;                   // offset of the mortar's points in n_hat/norm (lm1*lm2 points)
  int P[2][2], R[2][2];      // offsets of prolong/restrict matrices in the matrix pool, -1 if none
};

static __device__ __forceinline__ void nc_rotate_to_mortar(const MortarNC &M, const double *src, double *dst, int tid, int nt) {
  const int l1 = M.gs, l2 = M.gs;
  for (int t = tid; t < NV * l1 * l2; t += nt) {
    const int v = t / (l1 * l2), r = t - v * l1 * l2, i = r % l1, j = r / l1;
    int ni = i, nj = j;
    switch (M.orient) {
      case 3: ni = i; nj = l2 - 1 - j; break;
      case 2: ni = l1 - 1 - i; nj = l2 - 1 - j; break;
      case 1: ni = l1 - 1 - i; nj = j; break;
      case 4: ni = j; nj = i; break;
      case 5: ni = l2 - 1 - j; nj = i; break;
      case 6: ni = l2 - 1 - j; nj = l1 - 1 - i; break;
      case 7: ni = j; nj = l1 - 1 - i; break;
      default: break;
    }
    dst[v * NMX * NMX + nj * NMX + ni] = src[v * NMX * NMX + j * NMX + i];
  }
}
static __device__ __forceinline__ void nc_rotate_to_face(const MortarNC &M, const double *src, double *dst, int tid, int nt) {
  const int l1 = M.gs, l2 = M.gs;
  for (int t = tid; t < NV * l1 * l2; t += nt) {
    const int v = t / (l1 * l2), r = t - v * l1 * l2, i = r % l1, j = r / l1;
    int si = i, sj = j;
    switch (M.orient) {
      case 3: si = i; sj = l2 - 1 - j; break;
      case 2: si = l1 - 1 - i; sj = l2 - 1 - j; break;
      case 1: si = l1 - 1 - i; sj = j; break;
      case 4: si = j; sj = i; break;
      case 5: si = l2 - 1 - j; sj = i; break;
      case 6: si = l2 - 1 - j; sj = l1 - 1 - i; break;
      case 7: si = j; sj = l1 - 1 - i; break;
      default: break;
    }
    dst[v * NMX * NMX + j * NMX + i] = src[v * NMX * NMX + sj * NMX + si];
  }
}
// y = A[nout][nin] x along one direction of a [var][j][i] array (FMA chain)
static __device__ __forceinline__ double nc_apply(const double *A, int nin, int i, const double *x, int xs) {
  double acc = A[i * nin] * x[0];
  for (int k = 1; k < nin; ++k) acc = __fma_rn(A[i * nin + k], x[k * xs], acc);
  return acc;
}
// map_to_mortar_space: a (mortar orientation, face extents) -> mortar extents, in place via tmp
static __device__ void nc_to_mortar(const MortarNC &M, int side, const double *mats, double *a, double *tmp, int tid, int nt) {
  const bool c1 = M.conf[2 * side], c2 = M.conf[2 * side + 1];
  if (c1 && c2) return;
  const int n = side == 0 ? M.gm : M.gs;  // isotropic: len(idir) = len(jdir)
  if (!c1) {
    const double *A = mats + M.P[side][0];
    for (int t = tid; t < NV * n * M.lm1; t += nt) {
      const int v = t / (n * M.lm1), r = t - v * n * M.lm1, i = r % M.lm1, j = r / M.lm1;
      tmp[v * NMX * NMX + j * NMX + i] = nc_apply(A, n, i, a + v * NMX * NMX + j * NMX, 1);
    }
    __syncthreads();
    for (int t = tid; t < NV * n * M.lm1; t += nt) {
      const int v = t / (n * M.lm1), r = t - v * n * M.lm1, i = r % M.lm1, j = r / M.lm1;
      a[v * NMX * NMX + j * NMX + i] = tmp[v * NMX * NMX + j * NMX + i];
    }
    __syncthreads();
  }
  const int m1 = c1 ? n : M.lm1;
  if (!c2) {
    const double *A = mats + M.P[side][1];
    for (int t = tid; t < NV * m1 * M.lm2; t += nt) {
      const int v = t / (m1 * M.lm2), r = t - v * m1 * M.lm2, i = r % m1, j = r / m1;
      tmp[v * NMX * NMX + j * NMX + i] = nc_apply(A, n, j, a + v * NMX * NMX + i, NMX);
    }
    __syncthreads();
    for (int t = tid; t < NV * m1 * M.lm2; t += nt) {
      const int v = t / (m1 * M.lm2), r = t - v * m1 * M.lm2, i = r % m1, j = r / m1;
      a[v * NMX * NMX + j * NMX + i] = tmp[v * NMX * NMX + j * NMX + i];
    }
    __syncthreads();
  }
}
// map_to_face_space: mortar extents -> face extents (restriction), a -> out
static __device__ void nc_to_face(const MortarNC &M, int side, const double *mats, const double *a, double *out, double *tmp,
                           int tid, int nt) {
  const bool c1 = M.conf[2 * side], c2 = M.conf[2 * side + 1];
  for (int t = tid; t < NV * NMX * NMX; t += nt) out[t] = a[t];
  __syncthreads();
  if (c1 && c2) return;
  const int n = side == 0 ? M.gm : M.gs;
  if (!c1) {
    const double *A = mats + M.R[side][0];
    for (int t = tid; t < NV * M.lm2 * n; t += nt) {
      const int v = t / (M.lm2 * n), r = t - v * M.lm2 * n, i = r % n, j = r / n;
      tmp[v * NMX * NMX + j * NMX + i] = nc_apply(A, M.lm1, i, out + v * NMX * NMX + j * NMX, 1);
    }
    __syncthreads();
    for (int t = tid; t < NV * M.lm2 * n; t += nt) {
      const int v = t / (M.lm2 * n), r = t - v * M.lm2 * n, i = r % n, j = r / n;
      out[v * NMX * NMX + j * NMX + i] = tmp[v * NMX * NMX + j * NMX + i];
    }
    __syncthreads();
  }
  const int m1 = c1 ? M.lm1 : n;
  if (!c2) {
    const double *A = mats + M.R[side][1];
    for (int t = tid; t < NV * m1 * n; t += nt) {
      const int v = t / (m1 * n), r = t - v * m1 * n, i = r % m1, j = r / m1;
      tmp[v * NMX * NMX + j * NMX + i] = nc_apply(A, M.lm2, j, out + v * NMX * NMX + i, NMX);
    }
    __syncthreads();
    for (int t = tid; t < NV * m1 * n; t += nt) {
      const int v = t / (m1 * n), r = t - v * m1 * n, i = r % m1, j = r / m1;
      out[v * NMX * NMX + j * NMX + i] = tmp[v * NMX * NMX + j * NMX + i];
    }
    __syncthreads();
  }
}

static __global__ void __launch_bounds__(128) k_face_nc_inv(const MortarNC *__restrict__ mn, double *__restrict__ QF,
                                                     double *__restrict__ FF, const double *__restrict__ nh,
                                                     const double *__restrict__ nrm, const double *__restrict__ mats,
                                                     double gamma) {
  __shared__ double A1[NV * NMX * NMX], A2[NV * NMX * NMX], T0[NV * NMX * NMX], FL[NV * NMX * NMX],
      AV[NV * NMX * NMX];
  const MortarNC M = mn[blockIdx.x];
  const int tid = threadIdx.x, nt = blockDim.x;
  const int gm2 = M.gm * M.gm, gs2 = M.gs * M.gs;
  for (int t = tid; t < NV * NMX * NMX; t += nt) A1[t] = A2[t] = T0[t] = FL[t] = AV[t] = 0.0;
  __syncthreads();
  for (int t = tid; t < NV * gm2; t += nt) {
    const int v = t / gm2, p = t - v * gm2;
    A1[v * NMX * NMX + (p / M.gm) * NMX + p % M.gm] = QF[M.ms + t];
  }
  for (int t = tid; t < NV * gs2; t += nt) {
    const int v = t / gs2, p = t - v * gs2;
    T0[v * NMX * NMX + (p / M.gs) * NMX + p % M.gs] = QF[M.ss + t];
  }
  __syncthreads();
  if (M.orient) {
    nc_rotate_to_mortar(M, T0, A2, tid, nt);
  } else {
    for (int t = tid; t < NV * NMX * NMX; t += nt) A2[t] = T0[t];
  }
  __syncthreads();
  nc_to_mortar(M, 0, mats, A1, T0, tid, nt);
  nc_to_mortar(M, 1, mats, A2, T0, tid, nt);
  for (int t = tid; t < M.lm1 * M.lm2; t += nt) {
    const int i = t % M.lm1, j = t / M.lm1;
    double Q1[NV], Q2[NV], f[NV];
    for (int v = 0; v < NV; ++v) {
      Q1[v] = A1[v * NMX * NMX + j * NMX + i];
      Q2[v] = A2[v * NMX * NMX + j * NMX + i];
    }
    const long long gp = (long long)M.geo + t;
    const double n3[3] = {nh[gp * 3], nh[gp * 3 + 1], nh[gp * 3 + 2]};
    riemann(n3, nrm[gp], M.low ? Q2 : Q1, M.low ? Q1 : Q2, gamma, f);
    for (int v = 0; v < NV; ++v) {
      FL[v * NMX * NMX + j * NMX + i] = f[v];
      AV[v * NMX * NMX + j * NMX + i] = (Q1[v] + Q2[v]) * 0.5;
    }
  }
  __syncthreads();
  // master side: restrict flux and average, write face slots
  nc_to_face(M, 0, mats, FL, A1, T0, tid, nt);
  for (int t = tid; t < NV * gm2; t += nt) {
    const int v = t / gm2, p = t - v * gm2;
    FF[M.ms + t] = A1[v * NMX * NMX + (p / M.gm) * NMX + p % M.gm];
  }
  __syncthreads();
  nc_to_face(M, 0, mats, AV, A1, T0, tid, nt);
  for (int t = tid; t < NV * gm2; t += nt) {
    const int v = t / gm2, p = t - v * gm2;
    QF[M.ms + t] = A1[v * NMX * NMX + (p / M.gm) * NMX + p % M.gm];
  }
  __syncthreads();
  // slave side: restrict, rotate to the face, sign on the flux
  const double sgn = (double)M.sign;
  nc_to_face(M, 1, mats, FL, A1, T0, tid, nt);
  if (M.orient) {
    nc_rotate_to_face(M, A1, A2, tid, nt);
  } else {
    for (int t = tid; t < NV * NMX * NMX; t += nt) A2[t] = A1[t];
  }
  __syncthreads();
  for (int t = tid; t < NV * gs2; t += nt) {
    const int v = t / gs2, p = t - v * gs2;
    FF[M.ss + t] = sgn * A2[v * NMX * NMX + (p / M.gs) * NMX + p % M.gs];
  }
  __syncthreads();
  nc_to_face(M, 1, mats, AV, A1, T0, tid, nt);
  if (M.orient) {
    nc_rotate_to_face(M, A1, A2, tid, nt);
  } else {
    for (int t = tid; t < NV * NMX * NMX; t += nt) A2[t] = A1[t];
  }
  __syncthreads();
  for (int t = tid; t < NV * gs2; t += nt) {
    const int v = t / gs2, p = t - v * gs2;
    QF[M.ss + t] = A2[v * NMX * NMX + (p / M.gs) * NMX + p % M.gs];
  }
}

static __global__ void __launch_bounds__(128) k_face_nc_vis(const MortarNC *__restrict__ mn, double *__restrict__ VF,
                                                     const double *__restrict__ nrm, const double *__restrict__ mats) {
  __shared__ double R1[NV * NMX * NMX], R2[NV * NMX * NMX], T0[NV * NMX * NMX], QB[NV * NMX * NMX],
      T1[NV * NMX * NMX];
  const MortarNC M = mn[blockIdx.x];
  const int tid = threadIdx.x, nt = blockDim.x;
  const int gm2 = M.gm * M.gm, gs2 = M.gs * M.gs;
  const bool conf1 = M.conf[0] && M.conf[1], conf2 = M.conf[2] && M.conf[3];
  const double *nm = nrm + M.geo;  // mortar points, index i + lm1*j
  for (int t = tid; t < NV * NMX * NMX; t += nt) R1[t] = R2[t] = T0[t] = QB[t] = T1[t] = 0.0;
  __syncthreads();
  for (int t = tid; t < NV * gm2; t += nt) {
    const int v = t / gm2, p = t - v * gm2;
    R1[v * NMX * NMX + (p / M.gm) * NMX + p % M.gm] = VF[M.ms + t];
  }
  for (int t = tid; t < NV * gs2; t += nt) {
    const int v = t / gs2, p = t - v * gs2;
    R2[v * NMX * NMX + (p / M.gs) * NMX + p % M.gs] = VF[M.ss + t];
  }
  __syncthreads();
  // fv1: master side on mortar points
  if (!conf1) nc_to_mortar(M, 0, mats, R1, T0, tid, nt);
  for (int t = tid; t < NV * M.lm1 * M.lm2; t += nt) {
    const int v = t / (M.lm1 * M.lm2), r = t - v * M.lm1 * M.lm2, i = r % M.lm1, j = r / M.lm1;
    R1[v * NMX * NMX + j * NMX + i] = R1[v * NMX * NMX + j * NMX + i] / nm[i + M.lm1 * j];
  }
  __syncthreads();
  // fv2: slave side (conforming: divide in face indexing, then rotate)
  if (conf2) {
    for (int t = tid; t < NV * gs2; t += nt) {
      const int v = t / gs2, p = t - v * gs2, i = p % M.gs, j = p / M.gs;
      R2[v * NMX * NMX + j * NMX + i] = R2[v * NMX * NMX + j * NMX + i] / nm[i + M.lm1 * j];
    }
    __syncthreads();
    if (M.orient) {
      nc_rotate_to_mortar(M, R2, T1, tid, nt);
      __syncthreads();
      for (int t = tid; t < NV * NMX * NMX; t += nt) R2[t] = T1[t];
      __syncthreads();
    }
  } else {
    if (M.orient) {
      nc_rotate_to_mortar(M, R2, T1, tid, nt);
      __syncthreads();
      for (int t = tid; t < NV * NMX * NMX; t += nt) R2[t] = T1[t];
      __syncthreads();
    }
    nc_to_mortar(M, 1, mats, R2, T0, tid, nt);
    for (int t = tid; t < NV * M.lm1 * M.lm2; t += nt) {
      const int v = t / (M.lm1 * M.lm2), r = t - v * M.lm1 * M.lm2, i = r % M.lm1, j = r / M.lm1;
      R2[v * NMX * NMX + j * NMX + i] = R2[v * NMX * NMX + j * NMX + i] / nm[i + M.lm1 * j];
    }
    __syncthreads();
  }
  for (int t = tid; t < NV * M.lm1 * M.lm2; t += nt) {
    const int v = t / (M.lm1 * M.lm2), r = t - v * M.lm1 * M.lm2, i = r % M.lm1, j = r / M.lm1;
    double Qs = R2[v * NMX * NMX + j * NMX + i];
    if (M.nsign == -1) Qs = -Qs;
    const double Qm = R1[v * NMX * NMX + j * NMX + i];
    QB[v * NMX * NMX + j * NMX + i] = 0.5 * (Qm + Qs) * nm[i + M.lm1 * j];
  }
  __syncthreads();
  nc_to_face(M, 0, mats, QB, R1, T0, tid, nt);
  for (int t = tid; t < NV * gm2; t += nt) {
    const int v = t / gm2, p = t - v * gm2;
    VF[M.ms + t] = R1[v * NMX * NMX + (p / M.gm) * NMX + p % M.gm];
  }
  __syncthreads();
  if (M.sign == -1)
    for (int t = tid; t < NV * NMX * NMX; t += nt) QB[t] = -QB[t];
  __syncthreads();
  nc_to_face(M, 1, mats, QB, R1, T0, tid, nt);
  if (M.orient) {
    nc_rotate_to_face(M, R1, R2, tid, nt);
  } else {
    for (int t = tid; t < NV * NMX * NMX; t += nt) R2[t] = R1[t];
  }
  __syncthreads();
  for (int t = tid; t < NV * gs2; t += nt) {
    const int v = t / gs2, p = t - v * gs2;
    VF[M.ss + t] = R2[v * NMX * NMX + (p / M.gs) * NMX + p % M.gs];
  }
}

// ------------------------------------------------------------------ volume
struct VolArgs {
  const double *JQ;
  long long sq;
  const double *jac, *gg, *gm;  // metrics, layout per DIAG
  const double *muhg;           // [elem][G^3] entropy viscosity (EV)
  const double *nuhg;           // [elem][G^3] Smagorinsky viscosity (LES; null: off)
  const double *QF;             // [elem][6][5][G^2] averaged face state
  double *VF;                   // [elem][6][5][G^2] out: viscous normal flux at faces
  double *QTI;                  // [elem][5][G^3]   out: interior divergence sum
  double *EVB;                  // [elem][15][G^3]  out: gradients kept for EV / diagnostics
  Phys P;
  const int *ecase;             // optional: case of each element (ensembles)
  const double *rec;            // optional: per case {re, 1/re}
  int nel;                      // elements of the launch (set by the launcher)
};

template <int G, bool DIAG, bool EV, int SAVE> struct VolCfg {
  static constexpr int L = G + 1, NG = G * G * G, NL = L * G * G;
  static constexpr int NCH = DIAG ? 11 : 15;          // gradient fields interpolated to each grid
  static constexpr int NLB = EV ? 6 : 5;              // Lobatto slots (+ EV coefficient)
  static constexpr size_t MAXS = 232448;              // dynamic shared memory per CTA on sm_100
  static constexpr size_t bytes(bool pad, bool qsm) {
    return sizeof(double) *
           (size_t)(15 * NG + (NLB + NCH) * ((pad ? (L | 1) : L) * G * G) + (qsm ? 5 * NG : 0));
  }
  static constexpr bool QSM = bytes(false, true) <= MAXS;  // divergence sum kept in shared memory
  static constexpr bool PAD = QSM ? bytes(true, true) <= MAXS : bytes(true, false) <= MAXS;
  static constexpr int LX = PAD ? (L | 1) : L;        // x-grid line stride (odd: no bank conflicts)
  static constexpr int NLS = LX * G * G;              // stride of one field on a Lobatto grid
  static constexpr size_t SMEM = bytes(PAD, QSM);
  static constexpr int NT = G >= 8 ? DSEM_VOL_THREADS_P8 : 256;
};

// Line (a,b) of direction D on a Lobatto-grid array with x-stride LX.
template <int G, int LX, int D> __device__ __forceinline__ int lb_base(int a, int b) {
  return D == 0 ? LX * (a + G * b) : (D == 1 ? a + G * (G + 1) * b : a + G * b);
}
template <int G, int D> __device__ __forceinline__ constexpr int lb_stride() { return D == 0 ? 1 : (D == 1 ? G : G * G); }
template <int G, int D> __device__ __forceinline__ constexpr int g_stride() { return D == 0 ? 1 : (D == 1 ? G : G * G); }

// Interior Lobatto points of the 5 fields along D from q (Gauss layout); face
// points from the averaged face state.  Tasks [t0, t0 + 5*G^2) of a merged phase.
template <int G, int LX, int D>
__device__ __forceinline__ void build_task(int t, const double *q, const double *QF, double *LB, int NLS) {
  constexpr int L = G + 1, G2 = G * G, NG = G * G * G;
  const int v = t / G2, ln = t - v * G2, a = ln % G, b = ln / G;
  const double flo = QF[(face_lo(D) - 1) * 5 * G2 + v * G2 + ln];
  const double fhi = QF[(face_hi(D) - 1) * 5 * G2 + v * G2 + ln];
  double *y = LB + v * NLS + lb_base<G, LX, D>(a, b);
  constexpr int ys = lb_stride<G, D>();
  contract<G, false, 1, L - 1, 0, G>(q + v * NG + gbase<G>(D, a, b), g_stride<G, D>(), y, ys);
  y[0] = flo;
  y[(L - 1) * ys] = fhi;
}

// Derivative along D of Lobatto field f (f == 5: temperature, computed on the
// fly from the five fields, RHS.f90:66-83) and its contribution to the Gauss
// gradients (Gauss_Deriv, SolnDerivsc.f90:36-80).
template <int G, int LX, bool DIAG, int D>
__device__ __forceinline__ void deriv_task(int t, const double *LB, int NLS, const double *gg, double *GR, double *EVB,
                                           double gamma) {
  constexpr int L = G + 1, G2 = G * G, NG = G * G * G;
  const int f = t / G2, ln = t - f * G2, a = ln % G, b = ln / G;
  constexpr int ls = lb_stride<G, D>(), xs = g_stride<G, D>();
  const int l0 = lb_base<G, LX, D>(a, b);
  double w[G];
  if (f < 5) {
    contract_reg<G, true, 0, G, 0, L>(LB + f * NLS + l0, ls, w);
  } else {
    double T[L];
#pragma unroll
    for (int n = 0; n < L; ++n) {
      const int p = l0 + n * ls;
      const double q1 = LB[p], q2 = LB[NLS + p], q3 = LB[2 * NLS + p], q4 = LB[3 * NLS + p], q5 = LB[4 * NLS + p];
      const double r1 = 1.0 / q1, u = ddiv(q2, q1, r1), v = ddiv(q3, q1, r1), w = ddiv(q4, q1, r1);
      const double P = (gamma - 1.0) * (q5 - 0.5 * q1 * (u * u + v * v + w * w));
      T[n] = ddiv(P * gamma, q1, r1);
    }
    contract_reg<G, true, 0, G, 0, L>(T, 1, w);
  }
  const int p0 = gbase<G>(D, a, b);
  double *dst = f < 5 ? GR : EVB + 12 * NG;
  const int fo = f < 5 ? f * 3 : 0;
#pragma unroll
  for (int k = 0; k < G; ++k) {
    const int p = p0 + k * xs;
    if (DIAG) {
      dst[(fo + D) * NG + p] = gg[D * NG + p] * w[k];
    } else {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const double val = gg[p * 9 + D + 3 * c] * w[k];
        dst[(fo + c) * NG + p] = (D == 0) ? val : dst[(fo + c) * NG + p] + val;
      }
    }
  }
}

// Pass 2 for one direction: gradients to grid D, fluxes, interior divergence.
template <int G, bool DIAG, bool EV, int SAVE, int D>
__device__ __forceinline__ void vol_dir(const VolArgs &A, const double *JQ, const double *jac, const double *QF,
                                        const double *gm, const double *muhg, const double *GR, double *LB, double *CH,
                                        double *VF, double *QT, const Phys &P, int tid, int nt, long long &t_ph_) {
  using C = VolCfg<G, DIAG, EV, SAVE>;
  constexpr int L = G + 1, G2 = G * G, NG = G * G * G, NL = L * G * G;
  constexpr int LX = C::LX, NLS = C::NLS, NCH = C::NCH;
  constexpr int xs = g_stride<G, D>(), ls = lb_stride<G, D>();
  double *qpre = CH + 5 * NLS;  // state prefetched during the previous divergence phase
  if (D != 2) {
    for (int t = tid; t < 5 * G2; t += nt) build_task<G, LX, D>(t, qpre, QF, LB, NLS);
  }
  if (EV) {  // EV_Prolong (Prolong_gtol.f90:7-51)
    for (int t = tid; t < G2; t += nt) {
      const int a = t % G, b = t / G;
      contract<G, false, 0, L, 0, G>(muhg + gbase<G>(D, a, b), xs, LB + 5 * NLS + lb_base<G, LX, D>(a, b), ls);
    }
  }
  if (D != 2 || EV) __syncthreads();
  PHASE_MARK(8 + 4 * D);
  for (int t = tid; t < NCH * G2; t += nt) {  // gradients to grid D (Vis_Fluxes_new.f90:84-109)
    const int jf = t / G2, ln = t - jf * G2, a = ln % G, b = ln / G;
    const int src = DIAG ? diag_field(D, jf) : jf;
    contract<G, false, 0, L, 0, G>(GR + src * NG + gbase<G>(D, a, b), xs, CH + jf * NLS + lb_base<G, LX, D>(a, b), ls);
  }
  __syncthreads();
  PHASE_MARK(9 + 4 * D);
  for (int qi = tid; qi < NL; qi += nt) {  // fluxes on grid D (Vis_Fluxes_new.f90:115-228, fluxesH_newa.f90:276-352)
    int s, a, b, p, pg;
    if (D == 0) {
      s = qi % L;
      const int r = qi / L;
      a = r % G;
      b = r / G;
      p = s + LX * r;
      pg = qi;
    } else {
      ldecode<G>(D, qi, s, a, b);
      p = qi;
      pg = qi;
    }
    const double gdiag = DIAG ? gm[D * NL + pg] : 0.0;
    double Q[NV], Qx[NV], Qy[NV], Qz[NV], r[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) Q[v] = LB[v * NLS + p];
    const double rr = 1.0 / Q[0];
    double amu = 1.0;
    if (EV) amu = amu + LB[5 * NLS + p];
    const bool face = (s == 0 || s == L - 1);
    if (DIAG) {
      double c[11];
#pragma unroll
      for (int jf = 0; jf < 11; ++jf) c[jf] = CH[jf * NLS + p];
      double fl[NV];
      if (D == 0) {
        Qx[0] = c[0]; Qx[1] = c[1]; Qx[2] = c[2]; Qx[3] = c[3]; Qx[4] = c[4];
        Qy[0] = c[5]; Qy[1] = c[6]; Qy[2] = c[7]; Qy[3] = 0.0; Qy[4] = 0.0;
        Qz[0] = c[8]; Qz[1] = c[9]; Qz[3] = c[10]; Qz[2] = 0.0; Qz[4] = 0.0;
        vis_flux_x(Q, rr, Qx, Qy, Qz, amu, P, fl);
      } else if (D == 1) {
        Qy[0] = c[0]; Qy[1] = c[1]; Qy[2] = c[2]; Qy[3] = c[3]; Qy[4] = c[4];
        Qx[0] = c[5]; Qx[1] = c[6]; Qx[2] = c[7]; Qx[3] = 0.0; Qx[4] = 0.0;
        Qz[0] = c[8]; Qz[2] = c[9]; Qz[3] = c[10]; Qz[1] = 0.0; Qz[4] = 0.0;
        vis_flux_y(Q, rr, Qx, Qy, Qz, amu, P, fl);
      } else {
        Qz[0] = c[0]; Qz[1] = c[1]; Qz[2] = c[2]; Qz[3] = c[3]; Qz[4] = c[4];
        Qx[0] = c[5]; Qx[1] = c[6]; Qx[3] = c[7]; Qx[2] = 0.0; Qx[4] = 0.0;
        Qy[0] = c[8]; Qy[2] = c[9]; Qy[3] = c[10]; Qy[1] = 0.0; Qy[4] = 0.0;
        vis_flux_z(Q, rr, Qx, Qy, Qz, amu, P, fl);
      }
#pragma unroll
      for (int v = 0; v < NV; ++v) r[v] = gdiag * fl[v];
      if (face) {
        const int fc = s == 0 ? face_lo(D) : face_hi(D);
#pragma unroll
        for (int v = 0; v < NV; ++v) VF[(fc - 1) * 5 * G2 + v * G2 + a + G * b] = r[v];
      } else {
        double fi[NV];
        euler_flux(D, Q, rr, P.gamma, fi);
#pragma unroll
        for (int v = 0; v < NV; ++v) CH[v * NLS + p] = gdiag * fi[v] - ddiv(r[v], P.re, P.r_re);
      }
    } else {
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        Qx[v] = CH[(v * 3 + 0) * NLS + p];
        Qy[v] = CH[(v * 3 + 1) * NLS + p];
        Qz[v] = CH[(v * 3 + 2) * NLS + p];
      }
      double f[NV], g[NV], h[NV];
      vis_flux_x(Q, rr, Qx, Qy, Qz, amu, P, f);
      vis_flux_y(Q, rr, Qx, Qy, Qz, amu, P, g);
      vis_flux_z(Q, rr, Qx, Qy, Qz, amu, P, h);
      const double *g3 = gm + ((long long)D * NL + pg) * 3;
      const double m0 = g3[0], m1 = g3[1], m2 = g3[2];
#pragma unroll
      for (int v = 0; v < NV; ++v) r[v] = m0 * f[v] + m1 * g[v] + m2 * h[v];
      if (face) {
        const int fc = s == 0 ? face_lo(D) : face_hi(D);
#pragma unroll
        for (int v = 0; v < NV; ++v) VF[(fc - 1) * 5 * G2 + v * G2 + a + G * b] = r[v];
      } else {
        euler_fluxes3(Q, rr, P.gamma, f, g, h);
#pragma unroll
        for (int v = 0; v < NV; ++v) CH[v * NLS + p] = (m0 * f[v] + m1 * g[v] + m2 * h[v]) - ddiv(r[v], P.re, P.r_re);
      }
    }
  }
  __syncthreads();
  PHASE_MARK(10 + 4 * D);
  // interior divergence along D (updatea.f90:100-113), and the state for the next direction
  for (int t = tid; t < 5 * G2; t += nt) {
    const int v = t / G2, ln = t - v * G2, a = ln % G, b = ln / G;
    double S[G];
    contract_reg<G, true, 0, G, 1, L - 1>(CH + v * NLS + lb_base<G, LX, D>(a, b), ls, S);
    const int p0 = v * NG + gbase<G>(D, a, b);
#pragma unroll
    for (int k = 0; k < G; ++k) {
      const int p = p0 + k * xs;
      QT[p] = (D == 2) ? S[k] : QT[p] + S[k];
    }
  }
  if (D != 0) {
    for (int i = tid; i < 5 * NG; i += nt) qpre[i] = JQ[i] * jac[i % NG];
  }
  __syncthreads();
  PHASE_MARK(11 + 4 * D);
}

template <int G, bool DIAG, bool EV, int SAVE>
__global__ void __launch_bounds__(VolCfg<G, DIAG, EV, SAVE>::NT, 1) k_vol(VolArgs A) {
  using C = VolCfg<G, DIAG, EV, SAVE>;
  constexpr int G2 = G * G, NG = C::NG, NL = C::NL, LX = C::LX, NLS = C::NLS;
  extern __shared__ double sm[];
  double *GR = sm;
  double *LB = GR + 15 * NG;
  double *CH = LB + C::NLB * NLS;
  double *QTS = CH + C::NCH * NLS;  // divergence sum (when it fits)
  const int k = blockIdx.x, tid = threadIdx.x, nt = blockDim.x;
  const double *JQ = A.JQ + (long long)k * A.sq;
  const double *jac = A.jac + (long long)k * NG;
  const double *QF = A.QF + (long long)k * 30 * G2;
  double *VF = A.VF + (long long)k * 30 * G2;
  double *QTI = A.QTI + (long long)k * 5 * NG;
  double *QT = C::QSM ? QTS : QTI;
  double *EVB = SAVE ? A.EVB + (long long)k * 15 * NG : nullptr;
  const double *gg = A.gg + (long long)k * 3 * NG * (DIAG ? 1 : 3);
  const double *gm = A.gm + (long long)k * 3 * NL * (DIAG ? 1 : 3);
  const double *muhg = EV ? A.muhg + (long long)k * NG : nullptr;
  const double gamma = A.P.gamma;
  Phys P = A.P;
  if (A.rec) {  // per-case Reynolds number
    const int cs = A.ecase[k];
    P.re = A.rec[2 * cs];
    P.r_re = A.rec[2 * cs + 1];
  }
  long long t_ph_ = 0;
#ifdef DSEM_PHASE_TIMING
  t_ph_ = clock64();
#endif

  // Q*jacob (fluxesH_newa.f90:262-272)
  for (int i = tid; i < 5 * NG; i += nt) CH[i] = JQ[i] * jac[i % NG];
  __syncthreads();
  PHASE_MARK(0);
  // pass 1: Lobatto arrays and Gauss gradients, Lobatto array double-buffered
  double *LB2 = CH + 5 * NG;
  constexpr int NF = SAVE == 2 ? 6 : 5;
  for (int t = tid; t < 5 * G2; t += nt) build_task<G, LX, 0>(t, CH, QF, LB, NLS);
  __syncthreads();
  PHASE_MARK(1);
  for (int t = tid; t < (NF + 5) * G2; t += nt) {
    if (t < NF * G2)
      deriv_task<G, LX, DIAG, 0>(t, LB, NLS, gg, GR, EVB, gamma);
    else
      build_task<G, LX, 1>(t - NF * G2, CH, QF, LB2, NLS);
  }
  __syncthreads();
  PHASE_MARK(2);
  for (int t = tid; t < (NF + 5) * G2; t += nt) {
    if (t < NF * G2)
      deriv_task<G, LX, DIAG, 1>(t, LB2, NLS, gg, GR, EVB, gamma);
    else
      build_task<G, LX, 2>(t - NF * G2, CH, QF, LB, NLS);
  }
  __syncthreads();
  PHASE_MARK(3);
  for (int t = tid; t < NF * G2; t += nt) deriv_task<G, LX, DIAG, 2>(t, LB, NLS, gg, GR, EVB, gamma);
  __syncthreads();
  PHASE_MARK(4);
  if (SAVE) {
    for (int i = tid; i < 12 * NG; i += nt) EVB[i] = GR[i];
  }
  // pass 2: z (reusing the last Lobatto array), y, x
  vol_dir<G, DIAG, EV, SAVE, 2>(A, JQ, jac, QF, gm, muhg, GR, LB, CH, VF, QT, P, tid, nt, t_ph_);
  vol_dir<G, DIAG, EV, SAVE, 1>(A, JQ, jac, QF, gm, muhg, GR, LB, CH, VF, QT, P, tid, nt, t_ph_);
  vol_dir<G, DIAG, EV, SAVE, 0>(A, JQ, jac, QF, gm, muhg, GR, LB, CH, VF, QT, P, tid, nt, t_ph_);
  if (C::QSM) {
    for (int i = tid; i < 5 * NG; i += nt) QTI[i] = QTS[i];
  }
  PHASE_MARK(20);
}

// ------------------------------------------------------------------ update
struct UpdArgs {
  double *JQ, *gQ;
  long long sq;
  const double *jac;
  const double *QTI, *FF, *VF;
  double *QF;      // out: traces of the updated state
  double *JQo;     // optional: the updated state goes here and JQ is left unchanged
  double *Qt_out;  // optional: [elem][5][G^3]
  int *flag;       // bit 0: non-finite Qt
  double ark, cdt, re, r_re;  // r_re = 1/re
  int first, update;
  const int *ecase;           // optional: case of each element (ensembles)
  const double *rec, *dtc;    // optional: per case {re, 1/re} and dt; cdt = crk * dt
  double crk;
  // optional (k_update<G, true>): the BR1 average of the viscous face fluxes (k_face_vis)
  // done here from both sides' raw fluxes, so that no k_face_vis runs before.  fmc[6k + f]
  // is the conforming mortar on face f + 1 of element k, bit 8 of its flags set when that
  // face is the mortar's slave side; VFr is the base of the face slots its offsets index
  // (VF then holds raw fluxes) and vnrm the norms of its order's mortars.
  const MortarC *fmc;
  const double *VFr, *vnrm;
};

// BR1 average of one field at one mortar point (k_face_vis, send_flux_to_mortars) from the
// master's and the slave's raw viscous fluxes vm, vs and the mortar norms at the point and
// at its slave image: the value that the face on side `side` (0 master, 1 slave) receives,
// with k_face_vis's operations in k_face_vis's order.
__device__ __forceinline__ double vis_avg_point(const MortarC &M, int side, double vm, double vs, double nm_m,
                                                double nm_s) {
  const double rm = 1.0 / nm_m, rs = 1.0 / nm_s;
  const bool neg_n = (M.flags >> 4) & 1, neg_s = (M.flags >> 3) & 1;
  const double fv1 = ddiv(vm, nm_m, rm);
  const double fv2 = ddiv(vs, nm_s, rs);
  const double Qs = neg_n ? -fv2 : fv2;
  const double qb = 0.5 * (fv1 + Qs) * nm_m;
  return side ? (neg_s ? -qb : qb) : qb;
}

template <int G, bool FV = false> __global__ void __launch_bounds__(256) k_update(UpdArgs A) {
  constexpr int L = G + 1, G2 = G * G, NG = G * G * G;
  extern __shared__ double sm[];
  double *FB = sm;            // 30*G2 face fluxes
  double *QN = FB + 30 * G2;  // 5*NG updated physical Q
  double *Dlo = QN + 5 * NG;  // first and last columns of dmx
  double *Dhi = Dlo + G;
  const int k = blockIdx.x, tid = threadIdx.x, nt = blockDim.x;
  const double *FF = A.FF + (long long)k * 30 * G2;
  const double *VF = A.VF + (long long)k * 30 * G2;
  double re = A.re, rre = A.r_re, cdt = A.cdt;
  if (A.ecase) {
    const int cs = A.ecase[k];
    if (A.rec) {
      re = A.rec[2 * cs];
      rre = A.rec[2 * cs + 1];
    }
    if (A.dtc) cdt = A.crk * A.dtc[cs];
  }
  if constexpr (!FV) {
    // send_flux_to_faces_add; four items per thread in flight (HBM latency)
    for (int i0 = tid; i0 < 30 * G2; i0 += 4 * nt) {
      double ff[4], vf[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int i = i0 + u * nt;
        if (i < 30 * G2) {
          ff[u] = FF[i];
          vf[u] = VF[i];
        }
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int i = i0 + u * nt;
        if (i < 30 * G2) FB[i] = ff[u] - ddiv(vf[u], re, rre);
      }
    }
  } else {
    // the element's six mortars, then per item (face f, field v, mortar point pt) the
    // BR1 average of k_face_vis into this face's slot (pt on a master face, the point
    // sp that the orientation maps pt to on a slave face); four items per thread in flight
    __shared__ MortarC FM[6];
    if (tid < 6) FM[tid] = A.fmc[6LL * k + tid];
    __syncthreads();
    constexpr int UF = 4;
    for (int i0 = tid; i0 < 30 * G2; i0 += UF * nt) {
      double ff[UF], vm[UF], vs[UF], nm[UF], ns[UF];
      int own[UF];
#pragma unroll
      for (int u = 0; u < UF; ++u) {
        const int i = i0 + u * nt;
        own[u] = -1;
        if (i < 30 * G2) {
          const int f = i / (5 * G2), r = i - f * 5 * G2, v = r / G2, pt = r - v * G2;
          const MortarC &M = FM[f];
          int si, sj;
          slave_index<G>(M.flags & 7, pt % G, pt / G, si, sj);
          const int sp = si + G * sj;
          own[u] = f * 5 * G2 + v * G2 + (((M.flags >> 8) & 1) ? sp : pt);
          const long long g0 = (long long)M.geo * G2;
          ff[u] = FF[own[u]];
          vm[u] = A.VFr[M.ms + v * G2 + pt];
          vs[u] = A.VFr[M.ss + v * G2 + sp];
          nm[u] = A.vnrm[g0 + pt];
          ns[u] = A.vnrm[g0 + sp];
        }
      }
#pragma unroll
      for (int u = 0; u < UF; ++u) {
        if (own[u] < 0) continue;
        const MortarC &M = FM[own[u] / (5 * G2)];
        const double vf = vis_avg_point(M, (M.flags >> 8) & 1, vm[u], vs[u], nm[u], ns[u]);
        FB[own[u]] = ff[u] - ddiv(vf, re, rre);
      }
    }
  }
  for (int i = tid; i < G; i += nt) {
    Dlo[i] = Op<G>::D(i, 0);
    Dhi[i] = Op<G>::D(i, L - 1);
  }
  __syncthreads();
  double *JQ = A.JQ + (long long)k * A.sq;
  double *JQw = A.JQo ? A.JQo + (long long)k * A.sq : JQ;  // where the updated state goes
  double *gQ = A.gQ + (long long)k * A.sq;
  const double *QTI = A.QTI + (long long)k * 5 * NG;
  const double *jac = A.jac + (long long)k * NG;
  bool bad = false;
  constexpr int U = 2;  // items per thread with their loads in flight together
  for (int i0 = tid; i0 < 5 * NG; i0 += U * nt) {
    double qti[U], jq[U], gq[U], jc[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int i = i0 + u * nt;
      if (i < 5 * NG) {
        qti[u] = QTI[i];
        jq[u] = JQ[i];
        gq[u] = (A.update && !A.first) ? gQ[i] : 0.0;
        jc[u] = jac[i % NG];
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
    const int i = i0 + u * nt;
    if (i >= 5 * NG) break;
    const int v = i / NG, p = i - v * NG;
    const int n = p % G, m = (p / G) % G, l = p / G2;
    const double *F = FB + v * G2;
    double acc = qti[u];
    acc = __fma_rn(Dlo[n], F[5 * 5 * G2 + m + G * l], acc);  // face 6 (x = 0)
    acc = __fma_rn(Dhi[n], F[3 * 5 * G2 + m + G * l], acc);  // face 4 (x = 1)
    acc = __fma_rn(Dlo[m], F[0 * 5 * G2 + n + G * l], acc);  // face 1 (y = 0)
    acc = __fma_rn(Dhi[m], F[1 * 5 * G2 + n + G * l], acc);  // face 2 (y = 1)
    acc = __fma_rn(Dlo[l], F[2 * 5 * G2 + n + G * m], acc);  // face 3 (z = 0)
    acc = __fma_rn(Dhi[l], F[4 * 5 * G2 + n + G * m], acc);  // face 5 (z = 1)
    const double Qt = -acc;
    if (!isfinite(Qt)) bad = true;
    if (A.Qt_out) A.Qt_out[(long long)k * 5 * NG + i] = Qt;
    double q = jq[u];
    if (A.update) {  // updatea.f90:213-227
      const double g0 = A.first ? 0.0 : gq[u];
      const double g = A.ark * g0 + Qt;
      q = q + cdt * g;
      gQ[i] = g;
      JQw[i] = q;
    }
    QN[i] = q * jc[u];
    }
  }
  if (bad) atomicOr(A.flag, 1);
  __syncthreads();
  write_traces<G>(QN, A.QF + (long long)k * 30 * G2, tid, nt);
}

// --------------------------------------------------------------------- EV
struct EvArgs {
  const double *JQ;
  long long sq;
  const double *jac, *hd, *EVB;
  double *muhg;
  double *sens;  // optional: [elem][2][G^3] Ducros and density sensors for the Smagorinsky model
  int valid;
  Phys P;
  const int *ecase;   // optional: case of each element (ensembles)
  const double *rec;  // optional: per case {re, 1/re}
};

// RHS_ent_trans + Entropy_Viscosity at Gauss points (RHS.f90:21-278, EViscosity_GL.f90:19-101)
template <int G> __global__ void __launch_bounds__(256) k_ev(EvArgs A) {
  constexpr int NG = G * G * G;
  const int k = blockIdx.x;
  const double *JQ = A.JQ + (long long)k * A.sq;
  const double *jac = A.jac + (long long)k * NG;
  const double *hd = A.hd + (long long)k * NG;
  const double *EVB = A.EVB + (long long)k * 15 * NG;
  double *mu = A.muhg + (long long)k * NG;
  Phys P = A.P;
  if (A.rec) {
    const int cs = A.ecase[k];
    P.re = A.rec[2 * cs];
    P.r_re = A.rec[2 * cs + 1];
  }
  for (int p = threadIdx.x; p < NG; p += blockDim.x) {
    double out = 0.0;
    if (A.valid) {
      double Q[NV], Qx[NV], Qy[NV], Qz[NV], T1[3];
#pragma unroll
      for (int v = 0; v < NV; ++v) Q[v] = JQ[v * NG + p] * jac[p];
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        Qx[v] = EVB[(v * 3 + 0) * NG + p];
        Qy[v] = EVB[(v * 3 + 1) * NG + p];
        Qz[v] = EVB[(v * 3 + 2) * NG + p];
      }
      Qx[4] = Qy[4] = Qz[4] = 0.0;
      T1[0] = EVB[12 * NG + p];
      T1[1] = EVB[13 * NG + p];
      T1[2] = EVB[14 * NG + p];
      double duc;
      const double biS = ev_residual(P, Q, Qx, Qy, Qz, T1, duc);
      if (A.sens) {  // d%ducros, d%rhoSensor (RHS.f90:180-181)
        A.sens[(long long)k * 2 * NG + p] = duc;
        A.sens[(long long)k * 2 * NG + NG + p] = rho_sensor(Qx[0], Qy[0], Qz[0]);
      }
      const double rho = JQ[p] * jac[p];
      const double h = hd[p];
      double mur = P.cmu * P.re * rho * (h * h) * fabs(biS);
      if (P.ducros) mur = mur * duc;
      const double mx = mur >= 0.0 ? mur : 0.0;
      double m = mx <= P.mumax ? mx : P.mumax;
      if (!isfinite(m)) m = 0.0;
      out = m;
    }
    mu[p] = out;
  }
}

// ------------------------------------------------------------------- LES
struct LesArgs {
  const double *JQ;
  long long sq;
  const double *jac, *hd, *EVB;
  double *nuhg;
  const double *sens;  // [elem][2][G^3] Ducros and density sensors (k_ev; zero without entropy viscosity)
  int sensors;         // bit 0: shockSensor, bit 1: rhoSensor (staticSmag.f90:68-69)
  int valid;  // EVB holds the gradients of the last Fluxes call
  double re, cs, numax;
  const int *ecase;   // optional: case of each element (ensembles)
  const double *rec;  // optional: per case {re, 1/re}
};

// Static Smagorinsky viscosity at Gauss points (simpleSmag and filteredStrain,
// turbulence/staticSmago/staticSmag.f90:32-183): DSEM's rho = Q jacob(1,1,1)
// and velocities Q(2..4)/rho are kept as written; the optional shock and
// density sensors scale it (:68-69) with the values the step's entropy
// viscosity left (zero when it is off, as DSEM's zeroed arrays).
template <int G> __global__ void __launch_bounds__(128) k_les(LesArgs A) {
  constexpr int NG = G * G * G;
  const int k = blockIdx.x;
  const double *JQ = A.JQ + (long long)k * A.sq;
  const double *jac = A.jac + (long long)k * NG;
  const double *hd = A.hd + (long long)k * NG;
  const double *E = A.EVB + (long long)k * 15 * NG;
  double re = A.re;
  if (A.rec) re = A.rec[2 * A.ecase[k]];
  const double jac0 = jac[0];
  for (int p = threadIdx.x; p < NG; p += blockDim.x) {
    double gx[4] = {0.0, 0.0, 0.0, 0.0}, gy[4] = {0.0, 0.0, 0.0, 0.0}, gz[4] = {0.0, 0.0, 0.0, 0.0};
    if (A.valid) {
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        gx[v] = E[(v * 3 + 0) * NG + p];
        gy[v] = E[(v * 3 + 1) * NG + p];
        gz[v] = E[(v * 3 + 2) * NG + p];
      }
    }
    const double rho = JQ[p] * jac0;
    const double u = JQ[NG + p] / rho, v = JQ[2 * NG + p] / rho, w = JQ[3 * NG + p] / rho;
    const double rho_x = gx[0], rho_y = gy[0], rho_z = gz[0];
    const double u_x = (gx[1] - rho_x * u) / rho, u_y = (gy[1] - rho_y * u) / rho, u_z = (gz[1] - rho_z * u) / rho;
    const double v_x = (gx[2] - rho_x * v) / rho, v_y = (gy[2] - rho_y * v) / rho, v_z = (gz[2] - rho_z * v) / rho;
    const double w_x = (gx[3] - rho_x * w) / rho, w_y = (gy[3] - rho_y * w) / rho, w_z = (gz[3] - rho_z * w) / rho;
    const double S11 = u_x, S12 = 0.5 * (u_y + v_x), S13 = 0.5 * (u_z + w_x);
    const double S21 = 0.5 * (v_x + u_y), S22 = v_y, S23 = 0.5 * (v_z + w_y);
    const double S31 = 0.5 * (w_x + u_z), S32 = 0.5 * (w_y + v_z), S33 = w_z;
    const double S = sqrt(2.0 * S11 * S11 + 2.0 * S12 * S12 + 2.0 * S13 * S13 + 2.0 * S21 * S21 + 2.0 * S22 * S22 +
                          2.0 * S23 * S23 + 2.0 * S31 * S31 + 2.0 * S32 * S32 + 2.0 * S33 * S33);
    const double dg = hd[p];
    double nu = re * (A.cs * dg) * (A.cs * dg) * S;
    if (A.sensors & 1) nu = nu * (1.0 - A.sens[(long long)k * 2 * NG + p]);
    if (A.sensors & 2) nu = nu * A.sens[(long long)k * 2 * NG + NG + p];
    const double mx = nu >= 0.0 ? nu : 0.0;
    A.nuhg[(long long)k * NG + p] = mx <= A.numax ? mx : A.numax;
  }
}

}  // namespace dsem
