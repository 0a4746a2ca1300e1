// dsem_adjoint.cuh -- discrete adjoint of one right-hand side evaluation.
//
// Forward (one stage, dsem_stage.cuh / dsem_vol_diag.cuh):
//   q = JQ jacob -> face traces QFR -> mortars: Roe flux FF, averaged state QF
//   -> volume: Lobatto arrays, Gauss gradients, fluxes, interior divergence QTI,
//      viscous face flux VF -> BR1 average of VF -> Qt = -(QTI + face terms(FF - VF/Re)).
// Reverse, given lambda = dJ/dQt (LQT):
//   k_upd_adj       face terms           -> dJ/dFF (LFF); dJ/dVF after averaging is -LFF/Re
//   k_face_vis_adj  BR1 average          -> dJ/dVF before averaging (LVF)
//   k_vol_adj       volume (recomputed)  -> dJ/dJQ (LJQ), dJ/dQF averaged (LQF), dJ/d(1/Re)
//   k_face_inv_adj  Roe flux + average   -> dJ/dQFR (LQR)
//   k_trace_adj     face traces          -> LJQ += jacob * trace^T LQR
//                   (fused with the k_upd_adj of the stage reversed next)
// The volume adjoint can also add the gradient part of the derivative of the
// enstrophy-dissipation sum (energydissipation.f90:19-78) evaluated on the same
// gradients; k_eps_dir adds its direct part.  Entropy viscosity (without the
// Ducros sensor) enters through k_vol_adj<G, true> and k_ev_adj.
// Derivatives are exact up to rounding; every pointwise function is
// differentiated by hand-written reverse mode (riemann_dual / roe_vjp, the
// forward-mode derivative of the Roe flux, is kept as its independent check).
// Diagonal metrics and conforming mortars only.
#pragma once
#include <type_traits>

#include "dsem_stage.cuh"

namespace dsem {

// ------------------------------------------------------------ dual numbers
struct Dual {
  double v, d;
};
__device__ __forceinline__ Dual operator+(Dual a, Dual b) { return {a.v + b.v, a.d + b.d}; }
__device__ __forceinline__ Dual operator-(Dual a, Dual b) { return {a.v - b.v, a.d - b.d}; }
__device__ __forceinline__ Dual operator*(Dual a, Dual b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
__device__ __forceinline__ Dual operator/(Dual a, Dual b) {
  const double q = a.v / b.v;
  return {q, (a.d - q * b.d) / b.v};
}
__device__ __forceinline__ Dual operator+(Dual a, double b) { return {a.v + b, a.d}; }
__device__ __forceinline__ Dual operator+(double a, Dual b) { return {a + b.v, b.d}; }
__device__ __forceinline__ Dual operator-(Dual a, double b) { return {a.v - b, a.d}; }
__device__ __forceinline__ Dual operator-(double a, Dual b) { return {a - b.v, -b.d}; }
__device__ __forceinline__ Dual operator-(Dual a) { return {-a.v, -a.d}; }
__device__ __forceinline__ Dual operator*(Dual a, double b) { return {a.v * b, a.d * b}; }
__device__ __forceinline__ Dual operator*(double a, Dual b) { return {a * b.v, a * b.d}; }
__device__ __forceinline__ Dual operator/(Dual a, double b) { return {a.v / b, a.d / b}; }
__device__ __forceinline__ Dual operator/(double a, Dual b) {
  const double q = a / b.v;
  return {q, -q * b.d / b.v};
}
__device__ __forceinline__ Dual dsqrt(Dual a) {
  const double s = sqrt(a.v);
  return {s, a.d / (2.0 * s)};
}
__device__ __forceinline__ Dual dfabs(Dual a) { return a.v < 0.0 ? -a : a; }

// The Roe flux of riemann() (PhysLib.f90:231-320) on dual numbers; branches
// follow the values, as complex-step derivatives of the oracle do.
__device__ __forceinline__ void riemann_dual(const double *nh, double ds, const Dual *Ql, const Dual *Qr, double gamma,
                                             Dual *flux) {
  const Dual rho = Ql[0], rhou = Ql[1], rhov = Ql[2], rhow = Ql[3], rhoe = Ql[4];
  const Dual rhon = Qr[0], rhoun = Qr[1], rhovn = Qr[2], rhown = Qr[3], rhoen = Qr[4];
  const Dual ul = rhou / rho, vl = rhov / rho, wl = rhow / rho;
  const Dual pleft = (gamma - 1.0) * (rhoe - 0.5 / rho * (rhou * rhou + rhov * rhov + rhow * rhow));
  const Dual ur = rhoun / rhon, vr = rhovn / rhon, wr = rhown / rhon;
  const Dual pright = (gamma - 1.0) * (rhoen - 0.5 / rhon * (rhoun * rhoun + rhovn * rhovn + rhown * rhown));
  const Dual ql = nh[0] * ul + nh[1] * vl + nh[2] * wl;
  const Dual qr = nh[0] * ur + nh[1] * vr + nh[2] * wr;
  const Dual hl = 0.5 * (ul * ul + vl * vl + wl * wl) + gamma / (gamma - 1.0) * pleft / rho;
  const Dual hr = 0.5 * (ur * ur + vr * vr + wr * wr) + gamma / (gamma - 1.0) * pright / rhon;
  const Dual rtd = dsqrt(rho * rhon);
  const Dual betal = rho / (rho + rtd);
  const Dual betar = 1.0 - betal;
  const Dual utd = betal * ul + betar * ur;
  const Dual vtd = betal * vl + betar * vr;
  const Dual wtd = betal * wl + betar * wr;
  const Dual htd = betal * hl + betar * hr;
  const Dual atd2 = (gamma - 1.0) * (htd - 0.5 * (utd * utd + vtd * vtd + wtd * wtd));
  const Dual atd = dsqrt(atd2);
  const Dual qtd = utd * nh[0] + vtd * nh[1] + wtd * nh[2];
  if (qtd.v >= 0.0) {
    const Dual dw1 = 0.5 * ((pright - pleft) / atd2 - (qr - ql) * rtd / atd);
    const Dual sp1 = qtd - atd;
    const Dual sp1m = sp1.v <= 0.0 ? sp1 : Dual{0.0, 0.0};
    const Dual hd1m = ((gamma + 1.0) / 4.0 * atd / rtd) * dw1;
    const Dual e1 = -dfabs(sp1) - hd1m;
    const Dual eta1 = e1.v >= 0.0 ? e1 : Dual{0.0, 0.0};
    const Dual udw1 = dw1 * (sp1m - 0.5 * eta1);
    const Dual rql = rho * ql;
    flux[0] = ds * (rql + udw1);
    flux[1] = ds * (rql * ul + pleft * nh[0] + udw1 * (utd - atd * nh[0]));
    flux[2] = ds * (rql * vl + pleft * nh[1] + udw1 * (vtd - atd * nh[1]));
    flux[3] = ds * (rql * wl + pleft * nh[2] + udw1 * (wtd - atd * nh[2]));
    flux[4] = ds * (rql * hl + udw1 * (htd - qtd * atd));
  } else {
    const Dual dw4 = 0.5 * ((pright - pleft) / atd2 + (qr - ql) * rtd / atd);
    const Dual sp4 = qtd + atd;
    const Dual sp4p = sp4.v >= 0.0 ? sp4 : Dual{0.0, 0.0};
    const Dual hd4 = ((gamma + 1.0) / 4.0 * atd / rtd) * dw4;
    const Dual e4 = -dfabs(sp4) + hd4;
    const Dual eta4 = e4.v >= 0.0 ? e4 : Dual{0.0, 0.0};
    const Dual udw4 = dw4 * (sp4p + 0.5 * eta4);
    const Dual rqr = rhon * qr;
    flux[0] = ds * (rqr - udw4);
    flux[1] = ds * (rqr * ur + pright * nh[0] - udw4 * (utd + atd * nh[0]));
    flux[2] = ds * (rqr * vr + pright * nh[1] - udw4 * (vtd + atd * nh[1]));
    flux[3] = ds * (rqr * wr + pright * nh[2] - udw4 * (wtd + atd * nh[2]));
    flux[4] = ds * (rqr * hr - udw4 * (htd + qtd * atd));
  }
}

// lQl += (dF/dQl)^T lf, lQr += (dF/dQr)^T lf: one forward-mode pass per input.
__device__ __forceinline__ void roe_vjp(const double *nh, double ds, const double *Ql, const double *Qr, double gamma,
                                        const double *lf, double *lQl, double *lQr) {
#pragma unroll 1
  for (int j = 0; j < 10; ++j) {
    Dual L[NV], R[NV], F[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      L[v] = {Ql[v], j == v ? 1.0 : 0.0};
      R[v] = {Qr[v], j == NV + v ? 1.0 : 0.0};
    }
    riemann_dual(nh, ds, L, R, gamma, F);
    double s = 0.0;
#pragma unroll
    for (int v = 0; v < NV; ++v) s += lf[v] * F[v].d;
    if (j < NV)
      lQl[j] += s;
    else
      lQr[j - NV] += s;
  }
}

// Reverse mode of riemann(): lQl += (dF/dQl)^T lf, lQr += (dF/dQr)^T lf, the
// adjoint statements of each forward statement in reverse order; branches and
// kinks as riemann_dual (value of the forward quantity decides).
__device__ __forceinline__ void roe_vjp_rev(const double *nh, double ds, const double *Ql, const double *Qr,
                                            double gamma, const double *lfin, double *lQl, double *lQr) {
  const double g1 = gamma - 1.0, gg = gamma / (gamma - 1.0), K = (gamma + 1.0) / 4.0;
  const double rho = Ql[0], rhou = Ql[1], rhov = Ql[2], rhow = Ql[3], rhoe = Ql[4];
  const double rhon = Qr[0], rhoun = Qr[1], rhovn = Qr[2], rhown = Qr[3], rhoen = Qr[4];
  const double ul = rhou / rho, vl = rhov / rho, wl = rhow / rho;
  const double M2l = rhou * rhou + rhov * rhov + rhow * rhow;
  const double pleft = g1 * (rhoe - 0.5 / rho * M2l);
  const double ur = rhoun / rhon, vr = rhovn / rhon, wr = rhown / rhon;
  const double M2r = rhoun * rhoun + rhovn * rhovn + rhown * rhown;
  const double pright = g1 * (rhoen - 0.5 / rhon * M2r);
  const double ql = nh[0] * ul + nh[1] * vl + nh[2] * wl;
  const double qr = nh[0] * ur + nh[1] * vr + nh[2] * wr;
  const double hl = 0.5 * (ul * ul + vl * vl + wl * wl) + gg * pleft / rho;
  const double hr = 0.5 * (ur * ur + vr * vr + wr * wr) + gg * pright / rhon;
  const double rtd = sqrt(rho * rhon);
  const double sb = rho + rtd;
  const double betal = rho / sb, betar = 1.0 - betal;
  const double utd = betal * ul + betar * ur, vtd = betal * vl + betar * vr, wtd = betal * wl + betar * wr;
  const double htd = betal * hl + betar * hr;
  const double atd2 = g1 * (htd - 0.5 * (utd * utd + vtd * vtd + wtd * wtd));
  const double atd = sqrt(atd2);
  const double qtd = utd * nh[0] + vtd * nh[1] + wtd * nh[2];
  double lf[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) lf[v] = ds * lfin[v];
  const double lpn = lf[1] * nh[0] + lf[2] * nh[1] + lf[3] * nh[2];
  double lul = 0, lvl = 0, lwl = 0, lur = 0, lvr = 0, lwr = 0, lhl = 0, lhr = 0, lpl = 0, lpr = 0;
  double lutd = 0, lvtd = 0, lwtd = 0, lhtd = 0, latd = 0, lqtd = 0, lrho = 0, lrhon = 0, lql = 0, lqr = 0;
  double lrtd = 0, latd2 = 0, ldw = 0;
  const double X = (qr - ql) * rtd / atd;
  double lX = 0.0;
  if (qtd >= 0.0) {
    const double dw1 = 0.5 * ((pright - pleft) / atd2 - X);
    const double sp1 = qtd - atd;
    const double sp1m = sp1 <= 0.0 ? sp1 : 0.0;
    const double hd1m = (K * atd / rtd) * dw1;
    const double e1 = -fabs(sp1) - hd1m;
    const double eta1 = e1 >= 0.0 ? e1 : 0.0;
    const double udw1 = dw1 * (sp1m - 0.5 * eta1);
    const double rql = rho * ql;
    const double lrql = lf[0] + lf[1] * ul + lf[2] * vl + lf[3] * wl + lf[4] * hl;
    const double ludw = lf[0] + lf[1] * (utd - atd * nh[0]) + lf[2] * (vtd - atd * nh[1]) +
                        lf[3] * (wtd - atd * nh[2]) + lf[4] * (htd - qtd * atd);
    lul += lf[1] * rql;
    lvl += lf[2] * rql;
    lwl += lf[3] * rql;
    lhl += lf[4] * rql;
    lpl += lpn;
    lutd += lf[1] * udw1;
    lvtd += lf[2] * udw1;
    lwtd += lf[3] * udw1;
    lhtd += lf[4] * udw1;
    latd += -udw1 * lpn - lf[4] * udw1 * qtd;
    lqtd += -lf[4] * udw1 * atd;
    lrho += lrql * ql;
    lql += lrql * rho;
    ldw += ludw * (sp1m - 0.5 * eta1);
    const double lsp1m = ludw * dw1;
    const double leta = -0.5 * ludw * dw1;
    const double le = e1 >= 0.0 ? leta : 0.0;
    double lsp1 = -(sp1 < 0.0 ? -1.0 : 1.0) * le;
    const double lhd = -le;
    latd += K / rtd * dw1 * lhd;
    lrtd += -K * atd / (rtd * rtd) * dw1 * lhd;
    ldw += K * atd / rtd * lhd;
    lsp1 += sp1 <= 0.0 ? lsp1m : 0.0;
    lqtd += lsp1;
    latd -= lsp1;
    lpr += 0.5 / atd2 * ldw;
    lpl -= 0.5 / atd2 * ldw;
    latd2 += -0.5 * (pright - pleft) / (atd2 * atd2) * ldw;
    lX = -0.5 * ldw;
  } else {
    const double dw4 = 0.5 * ((pright - pleft) / atd2 + X);
    const double sp4 = qtd + atd;
    const double sp4p = sp4 >= 0.0 ? sp4 : 0.0;
    const double hd4 = (K * atd / rtd) * dw4;
    const double e4 = -fabs(sp4) + hd4;
    const double eta4 = e4 >= 0.0 ? e4 : 0.0;
    const double udw4 = dw4 * (sp4p + 0.5 * eta4);
    const double rqr = rhon * qr;
    const double lrqr = lf[0] + lf[1] * ur + lf[2] * vr + lf[3] * wr + lf[4] * hr;
    const double ludw = -(lf[0] + lf[1] * (utd + atd * nh[0]) + lf[2] * (vtd + atd * nh[1]) +
                          lf[3] * (wtd + atd * nh[2]) + lf[4] * (htd + qtd * atd));
    lur += lf[1] * rqr;
    lvr += lf[2] * rqr;
    lwr += lf[3] * rqr;
    lhr += lf[4] * rqr;
    lpr += lpn;
    lutd += -lf[1] * udw4;
    lvtd += -lf[2] * udw4;
    lwtd += -lf[3] * udw4;
    lhtd += -lf[4] * udw4;
    latd += -udw4 * lpn - lf[4] * udw4 * qtd;
    lqtd += -lf[4] * udw4 * atd;
    lrhon += lrqr * qr;
    lqr += lrqr * rhon;
    ldw += ludw * (sp4p + 0.5 * eta4);
    const double lsp4p = ludw * dw4;
    const double leta = 0.5 * ludw * dw4;
    const double le = e4 >= 0.0 ? leta : 0.0;
    double lsp4 = -(sp4 < 0.0 ? -1.0 : 1.0) * le;
    const double lhd = le;
    latd += K / rtd * dw4 * lhd;
    lrtd += -K * atd / (rtd * rtd) * dw4 * lhd;
    ldw += K * atd / rtd * lhd;
    lsp4 += sp4 >= 0.0 ? lsp4p : 0.0;
    lqtd += lsp4;
    latd += lsp4;
    lpr += 0.5 / atd2 * ldw;
    lpl -= 0.5 / atd2 * ldw;
    latd2 += -0.5 * (pright - pleft) / (atd2 * atd2) * ldw;
    lX = 0.5 * ldw;
  }
  // X = (qr - ql) rtd / atd
  lqr += lX * rtd / atd;
  lql -= lX * rtd / atd;
  lrtd += lX * (qr - ql) / atd;
  latd += -lX * X / atd;
  // qtd, atd, atd2
  lutd += nh[0] * lqtd;
  lvtd += nh[1] * lqtd;
  lwtd += nh[2] * lqtd;
  latd2 += latd / (2.0 * atd);
  lhtd += g1 * latd2;
  lutd += -g1 * utd * latd2;
  lvtd += -g1 * vtd * latd2;
  lwtd += -g1 * wtd * latd2;
  // Roe averages
  double lbl = hl * lhtd + ul * lutd + vl * lvtd + wl * lwtd;
  const double lbr = hr * lhtd + ur * lutd + vr * lvtd + wr * lwtd;
  lhl += betal * lhtd;
  lhr += betar * lhtd;
  lul += betal * lutd;
  lvl += betal * lvtd;
  lwl += betal * lwtd;
  lur += betar * lutd;
  lvr += betar * lvtd;
  lwr += betar * lwtd;
  lbl -= lbr;
  lrho += lbl * rtd / (sb * sb);
  lrtd += -lbl * rho / (sb * sb);
  lrho += lrtd * rhon / (2.0 * rtd);
  lrhon += lrtd * rho / (2.0 * rtd);
  // enthalpies
  lul += ul * lhl;
  lvl += vl * lhl;
  lwl += wl * lhl;
  lpl += gg / rho * lhl;
  lrho += -gg * pleft / (rho * rho) * lhl;
  lur += ur * lhr;
  lvr += vr * lhr;
  lwr += wr * lhr;
  lpr += gg / rhon * lhr;
  lrhon += -gg * pright / (rhon * rhon) * lhr;
  // normal velocities
  lul += nh[0] * lql;
  lvl += nh[1] * lql;
  lwl += nh[2] * lql;
  lur += nh[0] * lqr;
  lvr += nh[1] * lqr;
  lwr += nh[2] * lqr;
  // pressures
  lQl[4] += g1 * lpl;
  lrho += g1 * 0.5 * M2l / (rho * rho) * lpl;
  lQl[1] += -g1 * rhou / rho * lpl;
  lQl[2] += -g1 * rhov / rho * lpl;
  lQl[3] += -g1 * rhow / rho * lpl;
  lQr[4] += g1 * lpr;
  lrhon += g1 * 0.5 * M2r / (rhon * rhon) * lpr;
  lQr[1] += -g1 * rhoun / rhon * lpr;
  lQr[2] += -g1 * rhovn / rhon * lpr;
  lQr[3] += -g1 * rhown / rhon * lpr;
  // velocities
  lQl[1] += lul / rho;
  lQl[2] += lvl / rho;
  lQl[3] += lwl / rho;
  lrho += -(ul * lul + vl * lvl + wl * lwl) / rho;
  lQr[1] += lur / rhon;
  lQr[2] += lvr / rhon;
  lQr[3] += lwr / rhon;
  lrhon += -(ur * lur + vr * lvr + wr * lwr) / rhon;
  lQl[0] += lrho;
  lQr[0] += lrhon;
}

// ---------------------------------------------- hand-written reverse modes
// Euler flux along D (PhysLib.f90:17-124): lQ += (dF/dQ)^T lf.
template <int D> __device__ __forceinline__ void euler_vjp(const double *Q, double g, const double *lf, double *lQ) {
  const double rho = Q[0], ri = 1.0 / rho;
  const double vel[3] = {Q[1] * ri, Q[2] * ri, Q[3] * ri};
  const double S = vel[0] * vel[0] + vel[1] * vel[1] + vel[2] * vel[2];
  const double p = (g - 1.0) * (Q[4] - 0.5 * rho * S);
  double lvel[3] = {0.0, 0.0, 0.0}, lp = 0.0, lrho = 0.0;
  lQ[1 + D] += lf[0];
#pragma unroll
  for (int i = 0; i < 3; ++i) {  // f_{1+i} = Q[1+D] vel_i + delta_{iD} p
    lQ[1 + D] += vel[i] * lf[1 + i];
    lvel[i] += Q[1 + D] * lf[1 + i];
  }
  lp += lf[1 + D];
  lvel[D] += (Q[4] + p) * lf[4];  // f_4 = vel_D (rho e + p)
  lQ[4] += vel[D] * lf[4];
  lp += vel[D] * lf[4];
  lQ[4] += (g - 1.0) * lp;
  lrho += -(g - 1.0) * 0.5 * S * lp;
#pragma unroll
  for (int i = 0; i < 3; ++i) lvel[i] += -(g - 1.0) * rho * vel[i] * lp;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    lQ[1 + i] += lvel[i] * ri;
    lrho += -vel[i] * ri * lvel[i];
  }
  lQ[0] += lrho;
}

// Viscous flux along D (PhysLib.f90:419-583) with Gr[j][f] = d Q_f / d x_j:
// fv = the flux, lQ += (dF/dQ)^T lf, lG += (dF/dGr)^T lf; with lamu non-null,
// *lamu = (dF/d amu)^T lf (the entropy viscosity enters through amu = 1 + mu).
template <int D>
__device__ __forceinline__ void vis_vjp(const double *Q, const double (&Gr)[3][NV], double amu, const Phys &P,
                                        const double *lf, double *fv, double *lQ, double (&lG)[3][NV],
                                        double *lamu = nullptr) {
  const double g = P.gamma, rho = Q[0], ri = 1.0 / rho;
  const double vel[3] = {Q[1] * ri, Q[2] * ri, Q[3] * ri};
  const double S = vel[0] * vel[0] + vel[1] * vel[1] + vel[2] * vel[2];
  const double p = (g - 1.0) * (Q[4] - 0.5 * rho * S);
  double Gv[3][3];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) Gv[i][j] = (Gr[j][1 + i] - vel[i] * Gr[j][0]) * ri;
  const double div = Gv[0][0] + Gv[1][1] + Gv[2][2];
  const double vgD = vel[0] * Gv[0][D] + vel[1] * Gv[1][D] + vel[2] * Gv[2][D];
  const double pD = (g - 1.0) * (Gr[D][4] - 0.5 * Gr[D][0] * S - rho * vgD);
  const double K = P.mach * P.mach * g;
  const double A = pD - p * Gr[D][0] * ri;
  const double tD = A * K * ri;
  const double kap = 1.0 + (amu - 1.0) * 0.2 * P.r_gm1;
  const double rden = P.r_den;  // 1 / (pr mach^2 (gamma-1))
  double tau[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) tau[i] = amu * (Gv[i][D] + Gv[D][i]) - (i == D ? 2.0 / 3.0 * amu * div : 0.0);
  fv[0] = 0.0;
#pragma unroll
  for (int i = 0; i < 3; ++i) fv[1 + i] = tau[i];
  fv[4] = vel[0] * tau[0] + vel[1] * tau[1] + vel[2] * tau[2] + kap * tD * rden;
  // reverse
  const double l4 = lf[4];
  double lvel[3], ltau[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    lvel[i] = tau[i] * l4;
    ltau[i] = lf[1 + i] + vel[i] * l4;
  }
  const double ltD = kap * rden * l4;
  if (lamu) {  // tau_i = amu T_i; kap = 1 + (amu - 1) 0.2 / (gamma - 1)
    double la = l4 * 0.2 * P.r_gm1 * tD * rden;
#pragma unroll
    for (int i = 0; i < 3; ++i)
      la += ltau[i] * (Gv[i][D] + Gv[D][i] - (i == D ? 2.0 / 3.0 * div : 0.0));
    *lamu = la;
  }
  double lGv[3][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    lGv[i][D] += amu * ltau[i];
    lGv[D][i] += amu * ltau[i];
  }
  const double ldiv = -(2.0 / 3.0) * amu * ltau[D];
#pragma unroll
  for (int i = 0; i < 3; ++i) lGv[i][i] += ldiv;
  double lrho = 0.0, lp = 0.0, lS = 0.0;
  const double lA = K * ri * ltD;  // tD = A K / rho
  lrho += -tD * ri * ltD;
  const double lpD = lA;  // A = pD - p Gr[D][0] / rho
  lp += -Gr[D][0] * ri * lA;
  lG[D][0] += -p * ri * lA;
  lrho += p * Gr[D][0] * ri * ri * lA;
  lG[D][4] += (g - 1.0) * lpD;  // pD
  lG[D][0] += -(g - 1.0) * 0.5 * S * lpD;
  lS += -(g - 1.0) * 0.5 * Gr[D][0] * lpD;
  lrho += -(g - 1.0) * vgD * lpD;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    lvel[i] += -(g - 1.0) * rho * Gv[i][D] * lpD;
    lGv[i][D] += -(g - 1.0) * rho * vel[i] * lpD;
  }
#pragma unroll
  for (int i = 0; i < 3; ++i)  // Gv[i][j] = (Gr[j][1+i] - vel_i Gr[j][0]) / rho
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      if (!(i == D || j == D || i == j)) continue;  // lGv[i][j] is 0 there (the flux along D does not use it)
      const double l = lGv[i][j];
      lG[j][1 + i] += l * ri;
      lvel[i] += -Gr[j][0] * ri * l;
      lG[j][0] += -vel[i] * ri * l;
      lrho += -Gv[i][j] * ri * l;
    }
  lQ[4] += (g - 1.0) * lp;  // p
  lrho += -(g - 1.0) * 0.5 * S * lp;
  lS += -(g - 1.0) * 0.5 * rho * lp;
#pragma unroll
  for (int i = 0; i < 3; ++i) lvel[i] += 2.0 * vel[i] * lS;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    lQ[1 + i] += lvel[i] * ri;
    lrho += -vel[i] * ri * lvel[i];
  }
  lQ[0] += lrho;
}

// Enstrophy term of one Gauss point (energydissipation.f90:19-78, as k_diag):
// vort(JQ[0..3], gradients) ; lQ[0..3] += w dvort/dJQ, lgr[f*3+j] += w dvort/dgr.
__device__ __forceinline__ void vort_vjp(const double *Qj, double jc, const double *gr, double w, double *lQ,
                                         double *lgr) {
  const double Q1 = Qj[0];
  struct T3 {
    int a, b, g0;  // gradient field of the numerator, variable index, gradient field of rho
  };
  // udery, uderz, vderx, vderz, wderx, wdery
  const T3 t[6] = {{4, 1, 1}, {5, 1, 2}, {6, 2, 0}, {8, 2, 2}, {9, 3, 0}, {10, 3, 1}};
  double d[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) d[k] = (gr[t[k].a] - (Qj[t[k].b] / Q1) * gr[t[k].g0]) / Q1;
  const double c1 = (d[5] - d[3]) / jc, c2 = (d[1] - d[4]) / jc, c3 = (d[2] - d[0]) / jc;
  const double kk = 2.0 * w / jc;
  const double l1 = kk * c1 / jc, l2 = kk * c2 / jc, l3 = kk * c3 / jc;
  const double ld[6] = {-l3, l2, l3, -l1, -l2, l1};
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    const double Qb = Qj[t[k].b], G0 = gr[t[k].g0];
    lgr[t[k].a] += ld[k] / Q1;
    lgr[t[k].g0] += -Qb / (Q1 * Q1) * ld[k];
    lQ[t[k].b] += -G0 / (Q1 * Q1) * ld[k];
    lQ[0] += (Qb * G0 / (Q1 * Q1 * Q1) - d[k] / Q1) * ld[k];
  }
}

// ---------------------------------------------------------------- kernels
// Face terms of the divergence and the RK residual sign (k_update):
// ------------------------------------------------------------ boundary faces
// pow with a constant exponent on dual numbers
__device__ __forceinline__ Dual dpow(Dual a, double e) {
  const double pv = pow(a.v, e);
  return {pv, a.d * e * pow(a.v, e - 1.0)};
}

// wall_mirror, osher_flux and riemann_state (dsem_stage.cuh) on dual numbers,
// statement for statement; branches follow the values.
__device__ __forceinline__ void wall_mirror_dual(const double *nh, const Dual *Q1, Dual *Q2) {
  const Dual qnorm = nh[0] * Q1[1] + nh[1] * Q1[2] + nh[2] * Q1[3];
  const Dual tx = Q1[1] - qnorm * nh[0], ty = Q1[2] - qnorm * nh[1], tz = Q1[3] - qnorm * nh[2];
  Q2[0] = Q1[0];
  Q2[1] = tx - qnorm * nh[0];
  Q2[2] = ty - qnorm * nh[1];
  Q2[3] = tz - qnorm * nh[2];
  Q2[4] = Q1[4];
}

__device__ __noinline__ void osher_dual(const double *nh, double ds, const Dual *Ql, const Dual *Qr, double gamma,
                                        Dual *flux) {
  const double en1 = nh[0], en2 = nh[1], en3 = nh[2];
  const Dual rho = Ql[0], rhou = Ql[1], rhov = Ql[2], rhow = Ql[3], rhoe = Ql[4];
  const Dual rhon = Qr[0], rhoun = Qr[1], rhovn = Qr[2], rhown = Qr[3], rhoen = Qr[4];
  const Dual qdotn = (en1 * rhou + en2 * rhov + en3 * rhow) / rho;
  const Dual qdotnn = (en1 * rhoun + en2 * rhovn + en3 * rhown) / rhon;
  const Dual p = (gamma - 1.0) * (rhoe - 0.5 / rho * (rhou * rhou + rhov * rhov + rhow * rhow));
  const Dual a = dsqrt(gamma * p / rho);
  Dual pn = (gamma - 1.0) * (rhoen - 0.5 / rhon * (rhoun * rhoun + rhovn * rhovn + rhown * rhown));
  const Dual an = dsqrt(gamma * pn / rhon);
  const Dual q_tanx = rhoun / rhon - qdotnn * en1;
  const Dual q_tany = rhovn / rhon - qdotnn * en2;
  const Dual q_tanz = rhown / rhon - qdotnn * en3;
  const double z = (gamma - 1.0) / (2.0 * gamma);
  Dual Ha = -qdotnn / an + 2.0 / (gamma - 1.0);
  Ha = Ha / (qdotn / a + 2.0 / (gamma - 1.0));
  pn = p / dpow(Ha, 1.0 / z);
  Dual pstar = a + an - (qdotnn - qdotn) * ((gamma - 1.0) / 2.0);
  pstar = pstar / (a / dpow(p, z) + an / dpow(pn, z));
  pstar = dpow(pstar, 1.0 / z);
  Dual ustar = Ha * qdotn / a + qdotnn / an + 2.0 * (Ha - 1.0) / (gamma - 1.0);
  ustar = ustar / (Ha / a + 1.0 / an);
  const Dual rs = pstar * gamma / (an * an);
  const Dual u = q_tanx + en1 * ustar, v = q_tany + en2 * ustar, w = q_tanz + en3 * ustar;
  const Dual Q0 = rs, Q1 = rs * u, Q2 = rs * v, Q3 = rs * w;
  const Dual Q4 = pstar / (gamma - 1.0) + 0.5 * rs * (u * u + v * v + w * w);
  const Dual uu = Q1 / Q0, vv = Q2 / Q0, ww = Q3 / Q0;
  const Dual pp = (gamma - 1.0) * (Q4 - 0.5 * Q0 * (uu * uu + vv * vv + ww * ww));
  const Dual f[NV] = {Q1, pp + Q1 * uu, Q1 * vv, Q1 * ww, uu * (Q4 + pp)};
  const Dual g[NV] = {Q2, Q1 * vv, pp + Q2 * vv, Q3 * vv, vv * (Q4 + pp)};
  const Dual h[NV] = {Q3, Q1 * ww, Q2 * ww, pp + Q3 * ww, ww * (Q4 + pp)};
#pragma unroll
  for (int k = 0; k < NV; ++k) flux[k] = ds * (en1 * f[k] + en2 * g[k] + en3 * h[k]);
}

__device__ __noinline__ void riemann_state_dual(const double *nh, const Dual *Ql, const Dual *Qr, double gamma, Dual *Q) {
  const double en1 = nh[0], en2 = nh[1], en3 = nh[2];
  const Dual rho = Ql[0], rhou = Ql[1], rhov = Ql[2], rhow = Ql[3], rhoe = Ql[4];
  const Dual rhon = Qr[0], rhoun = Qr[1], rhovn = Qr[2], rhown = Qr[3], rhoen = Qr[4];
  const Dual qdotn = (en1 * rhou + en2 * rhov + en3 * rhow) / rho;
  const Dual qdotnn = (en1 * rhoun + en2 * rhovn + en3 * rhown) / rhon;
  const Dual p = (gamma - 1.0) * (rhoe - 0.5 / rho * (rhou * rhou + rhov * rhov + rhow * rhow));
  const Dual a = dsqrt(gamma * p / rho);
  const Dual pn = (gamma - 1.0) * (rhoen - 0.5 / rhon * (rhoun * rhoun + rhovn * rhovn + rhown * rhown));
  const Dual an = dsqrt(gamma * pn / rhon);
  const Dual e0 = 0.5 * (qdotn + qdotnn);
  const Dual eplus = e0 + 0.5 * (a + an);
  const Dual eminus = e0 - 0.5 * (a + an);
  Dual etos, q_tanx, q_tany, q_tanz;
  if (e0.v > 0.0) {
    etos = p / dpow(rho, gamma);
    q_tanx = rhou / rho - qdotn * en1;
    q_tany = rhov / rho - qdotn * en2;
    q_tanz = rhow / rho - qdotn * en3;
  } else {
    etos = pn / dpow(rhon, gamma);
    q_tanx = rhoun / rhon - qdotnn * en1;
    q_tany = rhovn / rhon - qdotnn * en2;
    q_tanz = rhown / rhon - qdotnn * en3;
  }
  const Dual rplus = eplus.v >= 0.0 ? qdotn + 2.0 / (gamma - 1.0) * a : qdotnn + 2.0 / (gamma - 1.0) * an;
  const Dual rminus = eminus.v >= 0.0 ? qdotn - 2.0 / (gamma - 1.0) * a : qdotnn - 2.0 / (gamma - 1.0) * an;
  const Dual qn = 0.5 * (rplus + rminus);
  const Dual as = 0.25 * (gamma - 1.0) * (rplus - rminus);
  const Dual rs = dpow(as * as / (gamma * etos), 1.0 / (gamma - 1.0));
  const Dual ps = dpow(rs, gamma) * etos;
  const Dual u = q_tanx + en1 * qn, v = q_tany + en2 * qn, w = q_tanz + en3 * qn;
  Q[0] = rs;
  Q[1] = rs * u;
  Q[2] = rs * v;
  Q[3] = rs * w;
  Q[4] = ps / (gamma - 1.0) + 0.5 * rs * (u * u + v * v + w * w);
}

// Inviscid boundary faces (k_face_bnd_inv), transposed: from dJ/dFF (LFF) and
// dJ/d(the face's Dirichlet state) (LQF) at each boundary point to dJ/d(its
// raw trace) (LQR).  One forward-mode pass per trace component, through the
// mirror state, the Roe or osher flux and the Dirichlet state.
template <int G>
__global__ void __launch_bounds__(128) k_face_bnd_inv_adj(const MortarB *__restrict__ mb, int nm,
                                                           const double *__restrict__ QFR,
                                                           const double *__restrict__ LFF,
                                                           const double *__restrict__ LQF, double *__restrict__ LQR,
                                                           const double *__restrict__ nh,
                                                           const double *__restrict__ nrm,
                                                           const double *__restrict__ qext, BndPhys P) {
  constexpr int G2 = G * G;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)nm * G2) return;
  const int m = (int)(t / G2), pt = (int)(t - (long long)m * G2);
  const MortarB M = mb[m];
  const int bc = M.flags & 7;
  const bool low = (M.flags >> 3) & 1;
  const long long gp = (long long)M.geo * G2 + pt;
  const double n3[3] = {nh[gp * 3], nh[gp * 3 + 1], nh[gp * 3 + 2]};
  const double ds = nrm[gp];
  double Q1[NV], lf[NV], lq[NV], Qx[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    Q1[v] = QFR[M.ms + v * G2 + pt];
    lf[v] = LFF[M.ms + v * G2 + pt];
    lq[v] = LQF[M.ms + v * G2 + pt];
    Qx[v] = (bc == BC_INFLOW || bc == BC_OUTFLOW) ? qext[(long long)M.geo * NV * G2 + v * G2 + pt] : 0.0;
  }
#pragma unroll 1
  for (int j = 0; j < NV; ++j) {
    Dual A[NV], B[NV], f[NV], qb[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) A[v] = {Q1[v], v == j ? 1.0 : 0.0};
    if (bc == BC_WALLADIAB || bc == BC_WALLISOTH) {
      wall_mirror_dual(n3, A, B);
      if (bc == BC_WALLADIAB) {
        riemann_dual(n3, ds, low ? B : A, low ? A : B, P.gamma, f);
        qb[4] = A[4];
      } else {
        const Dual rho = B[0];
        const Dual u = B[1] / rho, v = B[2] / rho, w = B[3] / rho;
        B[4] = (rho * P.twall) / P.cv + 0.5 * rho * (u * u + v * v + w * w);
        if (low) {
          const double mn[3] = {-n3[0], -n3[1], -n3[2]};
          osher_dual(mn, -ds, A, B, P.gamma, f);
        } else {
          osher_dual(n3, ds, A, B, P.gamma, f);
        }
        qb[4] = (A[0] * P.twall) / P.cv;
      }
      qb[0] = A[0];
      qb[1] = qb[2] = qb[3] = Dual{0.0, 0.0};
    } else {
#pragma unroll
      for (int v = 0; v < NV; ++v) B[v] = {Qx[v], 0.0};
      riemann_dual(n3, ds, low ? B : A, low ? A : B, P.gamma, f);
      riemann_state_dual(n3, low ? B : A, low ? A : B, P.gamma, qb);
    }
    double s = 0.0;
#pragma unroll
    for (int v = 0; v < NV; ++v) s += lf[v] * f[v].d + lq[v] * qb[v].d;
    LQR[M.ms + j * G2 + pt] = s;
  }
}

// Viscous boundary faces (k_face_bnd_vis), transposed: from dJ/dVF after the
// boundary condition (-LFF/Re) to dJ/dVF before it (LVF).  Inflow and outflow
// add the external flux (0.5 fv_ext |n|), whose 1/Re term the volume adjoint's
// Re * LVF . VF does not see: it goes to LRB, one slot per boundary point,
// accumulated over the sweep and summed at its end.
template <int G>
__global__ void __launch_bounds__(128) k_face_bnd_vis_adj(const MortarB *__restrict__ mb, int nm,
                                                           const double *__restrict__ LFF, double re,
                                                           double *__restrict__ LVF, const double *__restrict__ nrm,
                                                           const double *__restrict__ fvext, double *__restrict__ LRB) {
  constexpr int G2 = G * G;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)nm * G2) return;
  const int m = (int)(t / G2), pt = (int)(t - (long long)m * G2);
  const MortarB M = mb[m];
  const int bc = M.flags & 7;
  const bool neg_n = (M.flags >> 4) & 1;
  const long long gp = (long long)M.geo * G2 + pt;
  const double nm_m = nrm[gp];
  double lr = 0.0;
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    const double lb = -LFF[M.ms + v * G2 + pt] / re;  // dJ/d(boundary VF)
    double lfv1;
    if (bc == BC_WALLADIAB || bc == BC_WALLISOTH) {
      lfv1 = (v == 4 && bc == BC_WALLADIAB) ? 0.0 : lb * nm_m;
    } else {
      const double fx = fvext[(long long)M.geo * NV * G2 + v * G2 + pt];
      const double Qs = neg_n ? -fx : fx;
      lfv1 = 0.5 * nm_m * lb;
      lr += re * lb * (0.5 * Qs * nm_m);
    }
    LVF[M.ms + v * G2 + pt] = lfv1 / nm_m;
  }
  if (bc == BC_INFLOW || bc == BC_OUTFLOW) LRB[t] += lr;
}

// ------------------------------------------------- p-nonconforming mortars
// Transposes of the projections of k_face_nc_inv / k_face_nc_vis (dsem_stage.cuh:
// nc_to_mortar, nc_to_face, nc_rotate_to_*), on [var][j*NMX + i] arrays in shared memory.

// x[k] = sum_{i < nout} A[i*nin + k] y[i*ys]: the transpose of nc_apply
static __device__ __forceinline__ double nc_apply_t(const double *A, int nin, int nout, int k, const double *y, int ys) {
  double acc = A[k] * y[0];
  for (int i = 1; i < nout; ++i) acc = acc + A[i * nin + k] * y[i * ys];
  return acc;
}

// nc_to_mortar transposed: a (mortar extents) -> a (face extents), in place via tmp
static __device__ void nc_to_mortar_t(const MortarNC &M, int side, const double *mats, double *a, double *tmp, int tid,
                                      int nt) {
  const bool c1 = M.conf[2 * side], c2 = M.conf[2 * side + 1];
  if (c1 && c2) return;
  const int n = side == 0 ? M.gm : M.gs;
  const int m1 = c1 ? n : M.lm1;
  if (!c2) {  // the j step: out[j][i] = sum_k A[j*n + k] in[k][i], j < lm2, k < n, i < m1
    const double *A = mats + M.P[side][1];
    for (int t = tid; t < NV * m1 * n; t += nt) {
      const int v = t / (m1 * n), r = t - v * m1 * n, i = r % m1, k = r / m1;
      tmp[v * NMX * NMX + k * NMX + i] = nc_apply_t(A, n, M.lm2, k, a + v * NMX * NMX + i, NMX);
    }
    __syncthreads();
    for (int t = tid; t < NV * m1 * n; t += nt) {
      const int v = t / (m1 * n), r = t - v * m1 * n, i = r % m1, k = r / m1;
      a[v * NMX * NMX + k * NMX + i] = tmp[v * NMX * NMX + k * NMX + i];
    }
    __syncthreads();
  }
  if (!c1) {  // the i step: out[j][i] = sum_k A[i*n + k] in[j][k], i < lm1, j < n, k < n
    const double *A = mats + M.P[side][0];
    for (int t = tid; t < NV * n * n; t += nt) {
      const int v = t / (n * n), r = t - v * n * n, k = r % n, j = r / n;
      tmp[v * NMX * NMX + j * NMX + k] = nc_apply_t(A, n, M.lm1, k, a + v * NMX * NMX + j * NMX, 1);
    }
    __syncthreads();
    for (int t = tid; t < NV * n * n; t += nt) {
      const int v = t / (n * n), r = t - v * n * n, k = r % n, j = r / n;
      a[v * NMX * NMX + j * NMX + k] = tmp[v * NMX * NMX + j * NMX + k];
    }
    __syncthreads();
  }
}

// nc_to_face transposed: a (face extents) -> a (mortar extents), in place via tmp
static __device__ void nc_to_face_t(const MortarNC &M, int side, const double *mats, double *a, double *tmp, int tid,
                                    int nt) {
  const bool c1 = M.conf[2 * side], c2 = M.conf[2 * side + 1];
  if (c1 && c2) return;
  const int n = side == 0 ? M.gm : M.gs;
  const int m1 = c1 ? M.lm1 : n;
  if (!c2) {  // the j step: out[j][i] = sum_k R[j*lm2 + k] in[k][i], j < n, k < lm2, i < m1
    const double *A = mats + M.R[side][1];
    for (int t = tid; t < NV * m1 * M.lm2; t += nt) {
      const int v = t / (m1 * M.lm2), r = t - v * m1 * M.lm2, i = r % m1, k = r / m1;
      tmp[v * NMX * NMX + k * NMX + i] = nc_apply_t(A, M.lm2, n, k, a + v * NMX * NMX + i, NMX);
    }
    __syncthreads();
    for (int t = tid; t < NV * m1 * M.lm2; t += nt) {
      const int v = t / (m1 * M.lm2), r = t - v * m1 * M.lm2, i = r % m1, k = r / m1;
      a[v * NMX * NMX + k * NMX + i] = tmp[v * NMX * NMX + k * NMX + i];
    }
    __syncthreads();
  }
  if (!c1) {  // the i step: out[j][i] = sum_k R[i*lm1 + k] in[j][k], i < n, k < lm1, j < lm2
    const double *A = mats + M.R[side][0];
    for (int t = tid; t < NV * M.lm1 * M.lm2; t += nt) {
      const int v = t / (M.lm1 * M.lm2), r = t - v * M.lm1 * M.lm2, k = r % M.lm1, j = r / M.lm1;
      tmp[v * NMX * NMX + j * NMX + k] = nc_apply_t(A, M.lm1, n, k, a + v * NMX * NMX + j * NMX, 1);
    }
    __syncthreads();
    for (int t = tid; t < NV * M.lm1 * M.lm2; t += nt) {
      const int v = t / (M.lm1 * M.lm2), r = t - v * M.lm1 * M.lm2, k = r % M.lm1, j = r / M.lm1;
      a[v * NMX * NMX + j * NMX + k] = tmp[v * NMX * NMX + j * NMX + k];
    }
    __syncthreads();
  }
}

// face slot (var-major, n x n) <-> [var][j*NMX + i] array, with a factor on load
static __device__ __forceinline__ void nc_load(double *dst, const double *src, int n, double f, int tid, int nt) {
  for (int t = tid; t < NV * NMX * NMX; t += nt) dst[t] = 0.0;
  __syncthreads();
  const int n2 = n * n;
  for (int t = tid; t < NV * n2; t += nt) {
    const int v = t / n2, p = t - v * n2;
    dst[v * NMX * NMX + (p / n) * NMX + p % n] = f * src[t];
  }
  __syncthreads();
}
static __device__ __forceinline__ void nc_store(double *dst, const double *src, int n, int tid, int nt) {
  const int n2 = n * n;
  for (int t = tid; t < NV * n2; t += nt) {
    const int v = t / n2, p = t - v * n2;
    dst[t] = src[v * NMX * NMX + (p / n) * NMX + p % n];
  }
}
// b <- a (all of it); then a <- rotated b when the mortar has an orientation
static __device__ __forceinline__ void nc_rot_mortar_inplace(const MortarNC &M, double *a, double *b, int tid, int nt) {
  if (!M.orient) return;
  for (int t = tid; t < NV * NMX * NMX; t += nt) b[t] = 0.0;
  __syncthreads();
  nc_rotate_to_mortar(M, a, b, tid, nt);
  __syncthreads();
  for (int t = tid; t < NV * NMX * NMX; t += nt) a[t] = b[t];
  __syncthreads();
}
static __device__ __forceinline__ void nc_rot_face_inplace(const MortarNC &M, double *a, double *b, int tid, int nt) {
  if (!M.orient) return;
  for (int t = tid; t < NV * NMX * NMX; t += nt) b[t] = 0.0;
  __syncthreads();
  nc_rotate_to_face(M, a, b, tid, nt);
  __syncthreads();
  for (int t = tid; t < NV * NMX * NMX; t += nt) a[t] = b[t];
  __syncthreads();
}

// k_face_nc_inv transposed, one CTA per nonconforming mortar: from dJ/dFF (LFF) and dJ/d(the
// averaged state) (LQF) at both face slots to dJ/d(raw traces) (LQR).  The mortar-space states
// are recomputed from the raw traces QFR; rotations transpose to their inverses.
static __global__ void __launch_bounds__(128) k_face_nc_inv_adj(const MortarNC *__restrict__ mn,
                                                                 const double *__restrict__ QFR,
                                                                 const double *__restrict__ LFF,
                                                                 const double *__restrict__ LQF,
                                                                 double *__restrict__ LQR, const double *__restrict__ nh,
                                                                 const double *__restrict__ nrm,
                                                                 const double *__restrict__ mats, double gamma) {
  __shared__ double A1[NV * NMX * NMX], A2[NV * NMX * NMX], T0[NV * NMX * NMX], LF[NV * NMX * NMX],
      LA[NV * NMX * NMX], X[NV * NMX * NMX];
  const MortarNC M = mn[blockIdx.x];
  const int tid = threadIdx.x, nt = blockDim.x;
  // forward: the two sides' states on the mortar points
  nc_load(A1, QFR + M.ms, M.gm, 1.0, tid, nt);
  nc_load(A2, QFR + M.ss, M.gs, 1.0, tid, nt);
  nc_rot_mortar_inplace(M, A2, T0, tid, nt);
  nc_to_mortar(M, 0, mats, A1, T0, tid, nt);
  nc_to_mortar(M, 1, mats, A2, T0, tid, nt);
  // dJ/d(mortar flux) and dJ/d(mortar average) from both faces
  nc_load(LF, LFF + M.ms, M.gm, 1.0, tid, nt);
  nc_to_face_t(M, 0, mats, LF, T0, tid, nt);
  nc_load(X, LFF + M.ss, M.gs, (double)M.sign, tid, nt);
  nc_rot_mortar_inplace(M, X, T0, tid, nt);
  nc_to_face_t(M, 1, mats, X, T0, tid, nt);
  for (int t = tid; t < NV * NMX * NMX; t += nt) LF[t] += X[t];
  __syncthreads();
  nc_load(LA, LQF + M.ms, M.gm, 1.0, tid, nt);
  nc_to_face_t(M, 0, mats, LA, T0, tid, nt);
  nc_load(X, LQF + M.ss, M.gs, 1.0, tid, nt);
  nc_rot_mortar_inplace(M, X, T0, tid, nt);
  nc_to_face_t(M, 1, mats, X, T0, tid, nt);
  for (int t = tid; t < NV * NMX * NMX; t += nt) LA[t] += X[t];
  __syncthreads();
  // Roe flux and average at each mortar point, reversed; the states' adjoints replace them
  for (int t = tid; t < M.lm1 * M.lm2; t += nt) {
    const int i = t % M.lm1, j = t / M.lm1;
    double Q1[NV], Q2[NV], lf[NV], l1[NV], l2[NV];
    for (int v = 0; v < NV; ++v) {
      const int q = v * NMX * NMX + j * NMX + i;
      Q1[v] = A1[q];
      Q2[v] = A2[q];
      lf[v] = LF[q];
      l1[v] = 0.5 * LA[q];
      l2[v] = l1[v];
    }
    const long long gp = (long long)M.geo + t;
    const double n3[3] = {nh[gp * 3], nh[gp * 3 + 1], nh[gp * 3 + 2]};
    if (M.low)
      roe_vjp_rev(n3, nrm[gp], Q2, Q1, gamma, lf, l2, l1);
    else
      roe_vjp_rev(n3, nrm[gp], Q1, Q2, gamma, lf, l1, l2);
    for (int v = 0; v < NV; ++v) {
      const int q = v * NMX * NMX + j * NMX + i;
      A1[q] = l1[v];
      A2[q] = l2[v];
    }
  }
  __syncthreads();
  // back to the faces: prolongations transposed, the slave's rotation inverted
  nc_to_mortar_t(M, 0, mats, A1, T0, tid, nt);
  nc_store(LQR + M.ms, A1, M.gm, tid, nt);
  nc_to_mortar_t(M, 1, mats, A2, T0, tid, nt);
  nc_rot_face_inplace(M, A2, T0, tid, nt);
  nc_store(LQR + M.ss, A2, M.gs, tid, nt);
}

// k_face_nc_vis transposed: from dJ/dVF after the average (-LFF/Re at both faces) to dJ/dVF
// before it (LVF).
static __global__ void __launch_bounds__(128) k_face_nc_vis_adj(const MortarNC *__restrict__ mn,
                                                                 const double *__restrict__ LFF, double re,
                                                                 double *__restrict__ LVF,
                                                                 const double *__restrict__ nrm,
                                                                 const double *__restrict__ mats) {
  __shared__ double QB[NV * NMX * NMX], X[NV * NMX * NMX], T0[NV * NMX * NMX];
  const MortarNC M = mn[blockIdx.x];
  const int tid = threadIdx.x, nt = blockDim.x;
  const bool conf1 = M.conf[0] && M.conf[1], conf2 = M.conf[2] && M.conf[3];
  const double *nm = nrm + M.geo;  // mortar points, index i + lm1*j
  nc_load(QB, LFF + M.ms, M.gm, -1.0 / re, tid, nt);
  nc_to_face_t(M, 0, mats, QB, T0, tid, nt);
  nc_load(X, LFF + M.ss, M.gs, -1.0 / re, tid, nt);
  nc_rot_mortar_inplace(M, X, T0, tid, nt);
  nc_to_face_t(M, 1, mats, X, T0, tid, nt);
  const double sg = M.sign == -1 ? -1.0 : 1.0;
  for (int t = tid; t < NV * NMX * NMX; t += nt) QB[t] += sg * X[t];
  __syncthreads();
  // QB = 0.5 (fv1 + nsign fv2) |n| at the mortar points: dJ/dfv1 into QB, dJ/dfv2 into X
  for (int t = tid; t < NV * NMX * NMX; t += nt) X[t] = 0.0;
  __syncthreads();
  for (int t = tid; t < NV * M.lm1 * M.lm2; t += nt) {
    const int v = t / (M.lm1 * M.lm2), r = t - v * M.lm1 * M.lm2, i = r % M.lm1, j = r / M.lm1;
    const int q = v * NMX * NMX + j * NMX + i;
    const double l = 0.5 * nm[i + M.lm1 * j] * QB[q];
    QB[q] = l;
    X[q] = M.nsign == -1 ? -l : l;
  }
  __syncthreads();
  // master: fv1 = P0(VF) / |n|
  for (int t = tid; t < NV * M.lm1 * M.lm2; t += nt) {
    const int v = t / (M.lm1 * M.lm2), r = t - v * M.lm1 * M.lm2, i = r % M.lm1, j = r / M.lm1;
    QB[v * NMX * NMX + j * NMX + i] = QB[v * NMX * NMX + j * NMX + i] / nm[i + M.lm1 * j];
  }
  __syncthreads();
  if (!conf1) nc_to_mortar_t(M, 0, mats, QB, T0, tid, nt);
  nc_store(LVF + M.ms, QB, M.gm, tid, nt);
  // slave: conforming, fv2 = rotate(VF / |n| in face indexing); else fv2 = P1(rotate(VF)) / |n|
  if (conf2) {
    nc_rot_face_inplace(M, X, T0, tid, nt);
    for (int t = tid; t < NV * M.gs * M.gs; t += nt) {
      const int v = t / (M.gs * M.gs), r = t - v * M.gs * M.gs, i = r % M.gs, j = r / M.gs;
      X[v * NMX * NMX + j * NMX + i] = X[v * NMX * NMX + j * NMX + i] / nm[i + M.lm1 * j];
    }
    __syncthreads();
  } else {
    for (int t = tid; t < NV * M.lm1 * M.lm2; t += nt) {
      const int v = t / (M.lm1 * M.lm2), r = t - v * M.lm1 * M.lm2, i = r % M.lm1, j = r / M.lm1;
      X[v * NMX * NMX + j * NMX + i] = X[v * NMX * NMX + j * NMX + i] / nm[i + M.lm1 * j];
    }
    __syncthreads();
    nc_to_mortar_t(M, 1, mats, X, T0, tid, nt);
    nc_rot_face_inplace(M, X, T0, tid, nt);
  }
  nc_store(LVF + M.ss, X, M.gs, tid, nt);
}

// Qt = -(QTI + sum_faces D_edge FB), FB = FF - VF/Re, transposed for one element
// from its dJ/dQt (lam, shared) to dJ/dFF (LFF).  dJ/dVF is -LFF/Re, formed by
// k_face_vis_adj.
template <int G> __device__ __forceinline__ void face_terms_adj(const double *lam, int k, double *__restrict__ LFF) {
  constexpr int L = G + 1, G2 = G * G, NG = G * G * G;
  for (int t = threadIdx.x; t < 30 * G2; t += blockDim.x) {
    const int f = t / (5 * G2), r = t - f * 5 * G2, v = r / G2, ln = r - v * G2, i = ln % G, j = ln / G;
    const bool hi = (f == 1 || f == 3 || f == 4);
    double acc = 0.0;
#pragma unroll
    for (int n = 0; n < G; ++n) {
      int p;
      if (f == 3 || f == 5)  // faces 4, 6: lines along x at (m, l) = (i, j)
        p = n + G * (i + G * j);
      else if (f == 0 || f == 1)  // faces 1, 2: along y at (n, l)
        p = i + G * (n + G * j);
      else  // faces 3, 5: along z at (n, m)
        p = i + G * (j + G * n);
      const double dlo = Op<G>::D(n, 0), dhi = Op<G>::D(n, L - 1);
      acc += (hi ? dhi : dlo) * lam[v * NG + p];
    }
    LFF[(long long)k * 30 * G2 + t] = -acc;
  }
}

// The reverse sweep's first stage of a step: dJ/dQt += cdt dJ/dQ, then the face terms.
template <int G>
__global__ void __launch_bounds__(256) k_upd_adj(double *__restrict__ LQT, const double *__restrict__ LQ, double cdt,
                                                  double *__restrict__ LFF) {
  constexpr int NG = G * G * G;
  __shared__ double lam[5 * NG];  // this element's dJ/dQt after the RK step
  const int k = blockIdx.x;
  double *lamg = LQT + (long long)k * 5 * NG;
  const double *lq = LQ + (long long)k * 5 * NG;
  for (int i = threadIdx.x; i < 5 * NG; i += blockDim.x) {
    const double x = lamg[i] + cdt * lq[i];
    lamg[i] = x;
    lam[i] = x;
  }
  __syncthreads();
  face_terms_adj<G>(lam, k, LFF);
}

// BR1 average of the viscous normal flux (k_face_vis), transposed: from dJ/dVF
// after averaging (-LFF/Re) to dJ/dVF before it (LVF).
template <int G>
// With QFR non-null it also writes the averaged face states of k_face_inv into QF
// (as k_face_avg), from raw traces kept by the forward sweep.
__global__ void __launch_bounds__(128) k_face_vis_adj(const MortarC *__restrict__ mc, int nm,
                                                       const double *__restrict__ LFF, double re,
                                                       double *__restrict__ LVF, const double *__restrict__ nrm,
                                                       const double *__restrict__ QFR, double *__restrict__ QF) {
  constexpr int G2 = G * G;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)nm * G2) return;
  const int m = (int)(t / G2), pt = (int)(t - (long long)m * G2);
  const MortarC M = mc[m];
  int si, sj;
  slave_index<G>(M.flags & 7, pt % G, pt / G, si, sj);
  const int sp = si + G * sj;
  const long long g0 = (long long)M.geo * G2;
  const double nm_m = nrm[g0 + pt], nm_s = nrm[g0 + sp];
  const bool neg_n = (M.flags >> 4) & 1, neg_s = (M.flags >> 3) & 1;
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    const double lm = -LFF[M.ms + v * G2 + pt] / re, ls = -LFF[M.ss + v * G2 + sp] / re;
    const double lqb = lm + (neg_s ? -ls : ls);
    const double lh = 0.5 * nm_m * lqb;
    LVF[M.ms + v * G2 + pt] = lh / nm_m;
    LVF[M.ss + v * G2 + sp] = (neg_n ? -lh : lh) / nm_s;
  }
  if (QFR) {
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      const double avg = (QFR[M.ms + v * G2 + pt] + QFR[M.ss + v * G2 + sp]) * 0.5;
      QF[M.ms + v * G2 + pt] = avg;
      QF[M.ss + v * G2 + sp] = avg;
    }
  }
}

// Averaged face states of k_face_inv from raw traces kept by the forward sweep
// (the same expression; the Roe flux is not needed by the reverse sweep).
template <int G>
__global__ void __launch_bounds__(128) k_face_avg(const MortarC *__restrict__ mc, int nm, const double *__restrict__ QFR,
                                                   double *__restrict__ QF) {
  constexpr int G2 = G * G;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)nm * G2) return;
  const int m = (int)(t / G2), pt = (int)(t - (long long)m * G2);
  const MortarC M = mc[m];
  int si, sj;
  slave_index<G>(M.flags & 7, pt % G, pt / G, si, sj);
  const int sp = si + G * sj;
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    const double avg = (QFR[M.ms + v * G2 + pt] + QFR[M.ss + v * G2 + sp]) * 0.5;
    QF[M.ms + v * G2 + pt] = avg;
    QF[M.ss + v * G2 + sp] = avg;
  }
}

// Roe flux and averaged state (k_face_inv), transposed: QFR = raw traces.
template <int G>
__global__ void __launch_bounds__(128, 4) k_face_inv_adj(const MortarC *__restrict__ mc, int nm,
                                                       const double *__restrict__ QFR, const double *__restrict__ LFF,
                                                       const double *__restrict__ LQF, double *__restrict__ LQR,
                                                       const double *__restrict__ nh, const double *__restrict__ nrm,
                                                       double gamma) {
  constexpr int G2 = G * G;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)nm * G2) return;
  const int m = (int)(t / G2), pt = (int)(t - (long long)m * G2);
  const MortarC M = mc[m];
  int si, sj;
  slave_index<G>(M.flags & 7, pt % G, pt / G, si, sj);
  const int sp = si + G * sj;
  double Q1[NV], Q2[NV], lf[NV], l1[NV], l2[NV];
  const double sgn = ((M.flags >> 3) & 1) ? -1.0 : 1.0;
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    Q1[v] = QFR[M.ms + v * G2 + pt];
    Q2[v] = QFR[M.ss + v * G2 + sp];
    lf[v] = LFF[M.ms + v * G2 + pt] + sgn * LFF[M.ss + v * G2 + sp];
    const double la = 0.5 * (LQF[M.ms + v * G2 + pt] + LQF[M.ss + v * G2 + sp]);
    l1[v] = la;
    l2[v] = la;
  }
  const long long gp = (long long)M.geo * G2 + pt;
  const double n3[3] = {nh[gp * 3], nh[gp * 3 + 1], nh[gp * 3 + 2]};
  // one call with the operands ordered by the master face (no divergent copies)
  const bool low = (M.flags >> 5) & 1;
  double Ql[NV], Qr[NV], ll[NV], lr_[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    Ql[v] = low ? Q2[v] : Q1[v];
    Qr[v] = low ? Q1[v] : Q2[v];
    ll[v] = low ? l2[v] : l1[v];
    lr_[v] = low ? l1[v] : l2[v];
  }
  roe_vjp_rev(n3, nrm[gp], Ql, Qr, gamma, lf, ll, lr_);
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    LQR[M.ms + v * G2 + pt] = low ? lr_[v] : ll[v];
    LQR[M.ss + v * G2 + sp] = low ? ll[v] : lr_[v];
  }
}

// Face traces (write_traces), transposed: LJQ += jacob * trace^T LQR; then the
// RK step of the reverse sweep: dJ/dQ += LJQ, dJ/dQt *= ark.  With NEXT the
// first part of the stage before it in the reverse sweep follows in the same
// pass (k_upd_adj with cdt): dJ/dQt += cdt dJ/dQ and its face terms into LFF.
// The operations and their order are those of the two kernels run apart.
template <int G, bool NEXT>
__global__ void __launch_bounds__(256) k_trace_adj(const double *__restrict__ LQR, const double *__restrict__ jac,
                                                    const double *__restrict__ LJQ, double *__restrict__ LQ,
                                                    double *__restrict__ LQT, double ark, double cdt,
                                                    double *__restrict__ LFF) {
  constexpr int L = G + 1, G2 = G * G, NG = G * G * G;
  __shared__ double F[30 * G2];  // this element's face adjoints
  __shared__ double lam[NEXT ? 5 * NG : 1];  // its dJ/dQt after both RK steps
  __shared__ double b0[G], b1[G];  // end rows of the interpolation (thread-dependent index)
  const int k = blockIdx.x;
  for (int i = threadIdx.x; i < 30 * G2; i += blockDim.x) F[i] = LQR[(long long)k * 30 * G2 + i];
  if (threadIdx.x < G) {
    b0[threadIdx.x] = Op<G>::B(0, threadIdx.x);
    b1[threadIdx.x] = Op<G>::B(L - 1, threadIdx.x);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 5 * NG; i += blockDim.x) {
    const int v = i / NG, p = i - v * NG, n = p % G, m = (p / G) % G, l = p / G2;
    const double *Fv = F + v * G2;
    double s = b0[n] * Fv[5 * 5 * G2 + m + G * l];    // face 6 (x = 0)
    s += b1[n] * Fv[3 * 5 * G2 + m + G * l];          // face 4
    s += b0[m] * Fv[0 * 5 * G2 + n + G * l];          // face 1 (y = 0)
    s += b1[m] * Fv[1 * 5 * G2 + n + G * l];          // face 2
    s += b0[l] * Fv[2 * 5 * G2 + n + G * m];          // face 3 (z = 0)
    s += b1[l] * Fv[4 * 5 * G2 + n + G * m];          // face 5
    const long long o = (long long)k * 5 * NG + i;
    const double lq = LQ[o] + (LJQ[o] + jac[(long long)k * NG + p] * s);
    LQ[o] = lq;
    const double lt = LQT[o] * ark;
    if constexpr (NEXT) {
      const double x = lt + cdt * lq;
      LQT[o] = x;
      lam[i] = x;
    } else {
      LQT[o] = lt;
    }
  }
  if constexpr (NEXT) {
    __syncthreads();
    face_terms_adj<G>(lam, k, LFF);
  }
}

// Entropy viscosity at a step's start (k_ev: RHS_ent_trans and Entropy_Viscosity,
// RHS.f90:207-278, EViscosity_GL.f90:19-101), transposed:
// mu = min(max(cmu Re rho h^2 |D| [duc], 0), mumax) with D the entropy residual of
// ev_residual and, with the Ducros variant (shock = 3), its sensor duc.  From dJ/dmu (LMU) it adds
// dJ/dJQ of the step's start state into LQ and writes dJ/dEVB, the demand on
// the gradients saved by the previous step's last stage, into LEVB.
struct EvAdjArgs {
  const double *JQ, *jac, *hd, *EVB, *LMU;
  double *LQ, *LEVB;
  Phys P;
};

template <int G> __global__ void __launch_bounds__(128) k_ev_adj(EvAdjArgs A) {
  constexpr int NG = G * G * G;
  const int k = blockIdx.x;
  const double *JQ = A.JQ + (long long)k * 5 * NG;
  const double *jac = A.jac + (long long)k * NG;
  const double *hd = A.hd + (long long)k * NG;
  const double *E = A.EVB + (long long)k * 15 * NG;
  const Phys &P = A.P;
  const double g = P.gamma, g1 = P.gamma - 1.0;
  for (int p = threadIdx.x; p < NG; p += blockDim.x) {
    double Q[NV], Gq[3][4], T1[3];
#pragma unroll
    for (int v = 0; v < NV; ++v) Q[v] = JQ[v * NG + p] * jac[p];
#pragma unroll
    for (int v = 0; v < 4; ++v)
#pragma unroll
      for (int d = 0; d < 3; ++d) Gq[d][v] = E[(v * 3 + d) * NG + p];
#pragma unroll
    for (int d = 0; d < 3; ++d) T1[d] = E[(12 + d) * NG + p];
    // forward (as ev_residual)
    const double rho = Q[0], ri = 1.0 / rho;
    const double vel[3] = {Q[1] * ri, Q[2] * ri, Q[3] * ri};
    const double S = vel[0] * vel[0] + vel[1] * vel[1] + vel[2] * vel[2];
    const double pr = g1 * (Q[4] - 0.5 * rho * S);
    const double Tt = pr * g * ri;
    double Gv[3][3];  // d u_i / d x_j
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) Gv[i][j] = (Gq[j][1 + i] - vel[i] * Gq[j][0]) * ri;
    const double div = Gv[0][0] + Gv[1][1] + Gv[2][2];
    const double s01 = Gv[1][0] + Gv[0][1], s02 = Gv[0][2] + Gv[2][0], s12 = Gv[1][2] + Gv[2][1];
    const double phi = 2.0 * (Gv[0][0] * Gv[0][0] + Gv[1][1] * Gv[1][1] + Gv[2][2] * Gv[2][2]) +
                       (s01 * s01 + s02 * s02 + s12 * s12) - 2.0 * div * div / 3.0;
    const double t2 = T1[0] * T1[0] + T1[1] * T1[1] + T1[2] * T1[2];
    const double den = Tt * g1 * P.pr;
    const double gam = t2 / den;
    const double biS = ((phi + gam) / Tt) / P.re;
    const double h2 = hd[p] * hd[p];
    const double mur0 = P.cmu * P.re * rho * h2 * fabs(biS);
    // Ducros sensor (shock = 3): duc = min(max(div^2 / (div^2 + |curl|^2 + 1e-9), 0), 1)
    const double cw0 = Gv[2][1] - Gv[1][2], cw1 = Gv[0][2] - Gv[2][0], cw2 = Gv[1][0] - Gv[0][1];
    const double c2 = cw0 * cw0 + cw1 * cw1 + cw2 * cw2, d2 = div * div, den_r = d2 + c2 + 1.0e-9;
    const double rr = d2 / den_r;
    const double duc = P.ducros ? (rr >= 1.0 ? 1.0 : (rr <= 0.0 ? 0.0 : rr)) : 1.0;
    const double mur = P.ducros ? mur0 * duc : mur0;
    const bool active = isfinite(mur) && mur > 0.0 && mur < P.mumax;
    double lQ[NV] = {0.0, 0.0, 0.0, 0.0, 0.0}, lGq[3][4] = {}, lT1[3] = {0.0, 0.0, 0.0};
    if (active) {
      const double lmur_in = A.LMU[(long long)k * NG + p];
      const double lmur = P.ducros ? lmur_in * duc : lmur_in;  // d mur / d mur0
      double lrho = lmur * P.cmu * P.re * h2 * fabs(biS);
      const double lbiS = lmur * P.cmu * P.re * rho * h2 * (biS < 0.0 ? -1.0 : 1.0);
      const double lpg = lbiS / (Tt * P.re);  // d/d(phi + gam)
      double lTt = -lbiS * (phi + gam) / (Tt * Tt * P.re);
      // gam = t2 / (Tt (g - 1) Pr)
#pragma unroll
      for (int d = 0; d < 3; ++d) lT1[d] = lpg * 2.0 * T1[d] / den;
      lTt += -lpg * gam / Tt;
      // phi
      double lGv[3][3];
#pragma unroll
      for (int i = 0; i < 3; ++i) lGv[i][i] = lpg * (4.0 * Gv[i][i] - 4.0 * div / 3.0);
      lGv[1][0] = lGv[0][1] = lpg * 2.0 * s01;
      lGv[0][2] = lGv[2][0] = lpg * 2.0 * s02;
      lGv[1][2] = lGv[2][1] = lpg * 2.0 * s12;
      if (P.ducros && rr > 0.0 && rr < 1.0) {  // the sensor's share: mur = mur0 duc
        const double lr = lmur_in * mur0;
        const double ld2 = lr * (c2 + 1.0e-9) / (den_r * den_r), lc2 = -lr * d2 / (den_r * den_r);
        const double ldiv = ld2 * 2.0 * div;
#pragma unroll
        for (int i = 0; i < 3; ++i) lGv[i][i] += ldiv;
        lGv[2][1] += lc2 * 2.0 * cw0;
        lGv[1][2] -= lc2 * 2.0 * cw0;
        lGv[0][2] += lc2 * 2.0 * cw1;
        lGv[2][0] -= lc2 * 2.0 * cw1;
        lGv[1][0] += lc2 * 2.0 * cw2;
        lGv[0][1] -= lc2 * 2.0 * cw2;
      }
      double lvel[3] = {0.0, 0.0, 0.0};
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
          const double l = lGv[i][j];
          lGq[j][1 + i] += l * ri;
          lGq[j][0] += -vel[i] * ri * l;
          lvel[i] += -Gq[j][0] * ri * l;
          lrho += -Gv[i][j] * ri * l;
        }
      // Tt = p g / rho
      const double lp = lTt * g * ri;
      lrho += -lTt * Tt * ri;
      // p = (g - 1)(rho E - rho S / 2)
      lQ[4] += g1 * lp;
      lrho += -g1 * 0.5 * S * lp;
#pragma unroll
      for (int i = 0; i < 3; ++i) lvel[i] += -g1 * rho * vel[i] * lp;
      // vel_i = m_i / rho
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        lQ[1 + i] += lvel[i] * ri;
        lrho += -vel[i] * ri * lvel[i];
      }
      lQ[0] += lrho;
    }
    double *LQ = A.LQ + (long long)k * 5 * NG;
#pragma unroll
    for (int v = 0; v < NV; ++v) LQ[v * NG + p] += jac[p] * lQ[v];
    double *LE = A.LEVB + (long long)k * 15 * NG;
#pragma unroll
    for (int v = 0; v < 4; ++v)
#pragma unroll
      for (int d = 0; d < 3; ++d) LE[(v * 3 + d) * NG + p] = lGq[d][v];
#pragma unroll
    for (int d = 0; d < 3; ++d) LE[(12 + d) * NG + p] = lT1[d];
  }
}

// Smagorinsky viscosity at a step's start (k_les: simpleSmag, staticSmag.f90:191-201),
// transposed: nu = min(max(Re (Cs h)^2 |S|, 0), numax), |S| = sqrt(2 S_ij S_ij) from the
// velocity gradients of the gradients saved by the previous step's last stage.  From
// dJ/dnu (LNU) it adds dJ/dJQ of the step's start state into LQ, writes dJ/dEVB into
// LEVB (fields 12..14, the temperature gradients, get 0) and adds the element's
// dJ/d(1/Re) (nu depends on Re directly) into LR.  No shock or density sensor.
struct LesAdjArgs {
  const double *JQ, *jac, *hd, *EVB, *LNU;
  double *LQ, *LEVB, *LR;
  double re, cs, numax;
  int valid;  // the saved gradients existed (else nu = 0 and nothing flows back)
};

template <int G> __global__ void __launch_bounds__(128) k_les_adj(LesAdjArgs A) {
  constexpr int NG = G * G * G;
  const int k = blockIdx.x;
  const double *JQ = A.JQ + (long long)k * 5 * NG;
  const double *E = A.EVB + (long long)k * 15 * NG;
  const double jac0 = A.jac[(long long)k * NG];
  double *LQ = A.LQ + (long long)k * 5 * NG;
  double *LE = A.LEVB + (long long)k * 15 * NG;
  double lr = 0.0;
  for (int p = threadIdx.x; p < NG; p += blockDim.x) {
    double g[3][4] = {}, lg[3][4] = {}, lJ[4] = {0.0, 0.0, 0.0, 0.0};
    if (A.valid) {
#pragma unroll
      for (int v = 0; v < 4; ++v)
#pragma unroll
        for (int d = 0; d < 3; ++d) g[d][v] = E[(v * 3 + d) * NG + p];
      // forward, as k_les
      const double rho = JQ[p] * jac0;
      const double vel[3] = {JQ[NG + p] / rho, JQ[2 * NG + p] / rho, JQ[3 * NG + p] / rho};
      double V[3][3];  // V[i][d] = d vel_i / d x_d
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int d = 0; d < 3; ++d) V[i][d] = (g[d][1 + i] - g[d][0] * vel[i]) / rho;
      double Sm[3][3];
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) Sm[i][j] = i == j ? V[i][i] : 0.5 * (V[i][j] + V[j][i]);
      double X = 0.0;
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) X += 2.0 * Sm[i][j] * Sm[i][j];
      const double S = sqrt(X);
      const double dg = A.hd[(long long)k * NG + p];
      const double c2 = A.re * (A.cs * dg) * (A.cs * dg);
      const double nu = c2 * S;
      const double mx = nu >= 0.0 ? nu : 0.0;
      const double lnu = (nu >= 0.0 && mx <= A.numax) ? A.LNU[(long long)k * NG + p] : 0.0;
      lr += -lnu * A.re * nu;  // nu = Re (Cs h)^2 |S|: d nu / d(1/Re) = -Re nu
      if (S > 0.0 && lnu != 0.0) {
        const double lX = lnu * c2 * 0.5 / S;
        double lV[3][3];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
          for (int j = 0; j < 3; ++j) lV[i][j] = 0.0;
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
          for (int j = 0; j < 3; ++j) {
            const double lS = lX * 4.0 * Sm[i][j];
            if (i == j) {
              lV[i][i] += lS;
            } else {
              lV[i][j] += 0.5 * lS;
              lV[j][i] += 0.5 * lS;
            }
          }
        double lrho = 0.0, lvel[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
          for (int d = 0; d < 3; ++d) {
            const double l = lV[i][d];
            lg[d][1 + i] += l / rho;
            lg[d][0] += -l * vel[i] / rho;
            lvel[i] += -l * g[d][0] / rho;
            lrho += -l * V[i][d] / rho;
          }
#pragma unroll
        for (int i = 0; i < 3; ++i) {
          lJ[1 + i] += lvel[i] / rho;
          lrho += -lvel[i] * vel[i] / rho;
        }
        lJ[0] += lrho * jac0;
      }
    }
#pragma unroll
    for (int v = 0; v < 4; ++v) LQ[v * NG + p] += lJ[v];
#pragma unroll
    for (int v = 0; v < 4; ++v)
#pragma unroll
      for (int d = 0; d < 3; ++d) LE[(v * 3 + d) * NG + p] = lg[d][v];
#pragma unroll
    for (int d = 0; d < 3; ++d) LE[(12 + d) * NG + p] = 0.0;
  }
  // the element's dJ/d(1/Re): warp sums, then the four warps' sums in order
  __shared__ double red[4];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) lr += __shfl_xor_sync(0xffffffffu, lr, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = lr;
  __syncthreads();
  if (threadIdx.x == 0) A.LR[k] += red[0] + red[1] + red[2] + red[3];
}

struct VolAdjArgs {
  const double *JQ;
  const double *jac, *gg, *gm;  // diagonal metric layout
  const double *QF;             // averaged face state
  const double *LQT;            // dJ/dQt
  const double *LVF;            // dJ/dVF before averaging
  double *LJQ;                  // out: dJ/dJQ (volume part)
  double *LQF;                  // out: dJ/dQF (averaged face state)
  double *lr;                   // in/out: per element dJ/d(1/Re), accumulated over stages
  double eps_w;                 // weight of the enstrophy sum (0: none)
  const double *JQe;            // state whose JQ values the enstrophy sum uses (end of the step)
  int pf;                       // L2 prefetch distance in elements (the blocks resident at once), 0: none
  const double *muhg;           // entropy viscosity at the Gauss points (null: none)
  double *lmuhg;                // in/out with muhg: dJ/dmu at the Gauss points, accumulated over stages
  const double *levb;           // dJ/d(gradients this stage saved for the next step's viscosity), or null
  int les;                      // with muhg: it holds the Smagorinsky nu_t (amu = 1 + nu rho), not mu
  double *scr;                  // G >= 8: per element scratch of VolAdjCfg<G>::SCR doubles
  Phys P;
};


template <int G> struct VolAdjCfg {
  static constexpr int L = G + 1, G2 = G * G, NG = G * G * G, NL = L * G * G;
  // One element per SM (shared memory).  p <= 6: every array in shared memory, at least
  // one thread per Lobatto point of a grid.  p = 7, 8 (G >= 8): the element's working set
  // (471 KB at p = 8) is twice an SM's shared memory, so the Gauss gradients, their
  // adjoints and the interpolated-gradient adjoints (GLOB: 30 G^3 + 11 L G^2 doubles) live
  // in a per-element device scratch (L2-resident while the element runs), 512 threads.
  static constexpr bool GLOB = G >= 8;
  static constexpr int NT = GLOB ? 512 : (NL <= 256 ? 256 : ((NL + 31) / 32) * 32);
  static constexpr size_t SCR = GLOB ? (size_t)30 * NG + 11 * NL : 0;
  static constexpr size_t NDBL = 5 * NG + (GLOB ? 0 : 15 * NG + 15 * NG) + 5 * NL + 5 * NL + (GLOB ? 0 : 11 * NL) +
                                 5 * NG + 5 * NG + 30 * G2 + NT + 3 * NG + 30 * G2 + 2 * NG;
  static constexpr size_t SMEM = sizeof(double) * NDBL;
  static_assert(SMEM <= 227 * 1024, "one element's shared arrays must fit one CTA");
};

// Volume adjoint of one element (diagonal metrics): recomputes the Lobatto
// arrays and Gauss gradients, then runs the volume operations in reverse.
// EVK: the entropy-viscosity variant (muhg, lmuhg and levb used; otherwise ignored)
template <int G, bool EVK> __global__ void __launch_bounds__(VolAdjCfg<G>::NT, 1) k_vol_adj(VolAdjArgs A) {
  using C = VolAdjCfg<G>;
  constexpr int L = G + 1, G2 = G * G, NG = G * G * G, NL = L * G * G, NT = C::NT;
  extern __shared__ double sm[];
  double *q = sm;               // [5][NG] physical state
  double *GR, *LGR, *LG, *LB;
  if constexpr (C::GLOB) {
    double *x = A.scr + (long long)blockIdx.x * C::SCR;
    GR = x;
    LGR = x + 15 * NG;
    LG = x + 30 * NG;
    LB = q + 5 * NG;
  } else {
    GR = q + 5 * NG;   // [15][NG] Gauss gradients, field f*3 + direction
    LGR = GR + 15 * NG;  // [15][NG] their adjoints
    LB = LGR + 15 * NG;  // [5][NL] Lobatto arrays of the current grid
  }
  double *LL = LB + 5 * NL;     // [5][NL] their adjoints
  if constexpr (!C::GLOB) LG = LL + 5 * NL;  // [11][NL] adjoints of the interpolated gradient fields
  double *LQ = LL + 5 * NL + (C::GLOB ? 0 : 11 * NL);  // [5][NG] dJ/dq
  double *LAM = LQ + 5 * NG;    // [5][NG] dJ/dQt
  double *LQFs = LAM + 5 * NG;  // [30][G2] dJ/dQF
  double *red = LQFs + 30 * G2;  // [NT]
  double *gg = red + NT;         // [3][NG] metric diagonal at the Gauss points
  double *QF = gg + 3 * NG;      // [30][G2] averaged face states
  double *MU = QF + 30 * G2;     // [NG] entropy viscosity (EV runs)
  double *LMU = MU + NG;         // [NG] its adjoint
  const int k = blockIdx.x, tid = threadIdx.x;
  const double *JQ = A.JQ + (long long)k * 5 * NG;
  const double *jac = A.jac + (long long)k * NG;
  const double *ggk = A.gg + (long long)k * 3 * NG;
  const double *gm = A.gm + (long long)k * 3 * NL;
  const double *QFk = A.QF + (long long)k * 30 * G2;
  const double *LVF = A.LVF + (long long)k * 30 * G2;
  double *LJQ = A.LJQ + (long long)k * 5 * NG;
  const Phys P = A.P;
  const double gamma = P.gamma;
  double lr = 0.0;
  long long t_ph_ = 0;
  (void)t_ph_;
#ifdef DSEM_PHASE_TIMING
  t_ph_ = clock64();
#endif
  // the element that starts about one wave of blocks later: its inputs into L2
  if (A.pf > 0 && k + A.pf < (int)gridDim.x) {
    const long long n = k + A.pf;
    prefetch_l2(A.JQ + n * 5 * NG, 5 * NG, tid, NT);
    prefetch_l2(A.LQT + n * 5 * NG, 5 * NG, tid, NT);
    prefetch_l2(A.jac + n * NG, NG, tid, NT);
    prefetch_l2(A.gg + n * 3 * NG, 3 * NG, tid, NT);
    prefetch_l2(A.QF + n * 30 * G2, 30 * G2, tid, NT);
    prefetch_l2(A.gm + n * 3 * NL, 3 * NL, tid, NT);
    prefetch_l2(A.LVF + n * 30 * G2, 30 * G2, tid, NT);
  }

  {  // state, dJ/dQt, metrics and face states: all of a thread's loads in flight at once
    constexpr int NQ = (5 * NG + NT - 1) / NT, NM = (3 * NG + NT - 1) / NT, NF = (30 * G2 + NT - 1) / NT;
    const double *lqt = A.LQT + (long long)k * 5 * NG;
    double qv[NQ], jv[NQ], lv[NQ], mv[NM], fv[NF];
#pragma unroll
    for (int j = 0; j < NQ; ++j) {
      const int i = tid + j * NT;
      if (i < 5 * NG) {
        qv[j] = JQ[i];
        jv[j] = jac[i % NG];
        lv[j] = lqt[i];
      }
    }
#pragma unroll
    for (int j = 0; j < NM; ++j)
      if (tid + j * NT < 3 * NG) mv[j] = ggk[tid + j * NT];
#pragma unroll
    for (int j = 0; j < NF; ++j)
      if (tid + j * NT < 30 * G2) fv[j] = QFk[tid + j * NT];
#pragma unroll
    for (int j = 0; j < NQ; ++j) {
      const int i = tid + j * NT;
      if (i < 5 * NG) {
        q[i] = qv[j] * jv[j];
        LAM[i] = lv[j];
        LQ[i] = 0.0;
      }
    }
#pragma unroll
    for (int j = 0; j < NM; ++j)
      if (tid + j * NT < 3 * NG) gg[tid + j * NT] = mv[j];
#pragma unroll
    for (int j = 0; j < NF; ++j)
      if (tid + j * NT < 30 * G2) QF[tid + j * NT] = fv[j];
  }
  // LGR starts from the next step's demand on the gradients this stage saves
  // (fields 0..3: EVB has the same layout as GR); the energy gradients start at 0
  if constexpr (EVK) {
    for (int i = tid; i < 15 * NG; i += NT) LGR[i] = (A.levb && i < 12 * NG) ? A.levb[(long long)k * 15 * NG + i] : 0.0;
    for (int i = tid; i < NG; i += NT) {
      MU[i] = A.muhg[(long long)k * NG + i];
      LMU[i] = 0.0;
    }
  } else {
    for (int i = tid; i < 15 * NG; i += NT) LGR[i] = 0.0;
  }
  for (int i = tid; i < 30 * G2; i += NT) LQFs[i] = 0.0;
  __syncthreads();
  PHASE_MARK(21);

  // ---- forward: Gauss gradients of the five fields, one task per (direction, field, line):
  // the Lobatto line is built and differentiated in registers
  auto grad_task = [&](auto Dc, int f, int ln) {
    constexpr int D = decltype(Dc)::value;
    constexpr int xs = D == 0 ? 1 : (D == 1 ? G : G2);
    const int a = ln % G, b = ln / G;
    const int p0 = gbase<G>(D, a, b);
    double x[G], y[L];
#pragma unroll
    for (int kk = 0; kk < G; ++kk) x[kk] = q[f * NG + p0 + kk * xs];
    y[0] = QF[(face_lo(D) - 1) * 5 * G2 + f * G2 + ln];
    y[L - 1] = QF[(face_hi(D) - 1) * 5 * G2 + f * G2 + ln];
#pragma unroll
    for (int s = 1; s < L - 1; ++s) {
      double acc = Op<G>::B(s, 0) * x[0];
#pragma unroll
      for (int kk = 1; kk < G; ++kk) acc = __fma_rn(Op<G>::B(s, kk), x[kk], acc);
      y[s] = acc;
    }
#pragma unroll
    for (int kk = 0; kk < G; ++kk) {
      double acc = Op<G>::D(kk, 0) * y[0];
#pragma unroll
      for (int s = 1; s < L; ++s) acc = __fma_rn(Op<G>::D(kk, s), y[s], acc);
      GR[(f * 3 + D) * NG + p0 + kk * xs] = gg[D * NG + p0 + kk * xs] * acc;
    }
  };
  for (int t = tid; t < 15 * G2; t += NT) {
    const int df = t / G2, ln = t - df * G2, D = df / 5, f = df - D * 5;
    if (D == 0)
      grad_task(std::integral_constant<int, 0>{}, f, ln);
    else if (D == 1)
      grad_task(std::integral_constant<int, 1>{}, f, ln);
    else
      grad_task(std::integral_constant<int, 2>{}, f, ln);
  }
  __syncthreads();
  PHASE_MARK(22);

  // ---- enstrophy term (energydissipation.f90:19-78) on these gradients and the
  // JQ values of JQe: its gradient part, into LGR (the JQe part: k_eps_dir)
  if (A.eps_w != 0.0) {
    const double *JQe = A.JQe + (long long)k * 5 * NG;
    for (int p = tid; p < NG; p += NT) {
      double Qj[4], gr[12], lgr[12], lq4[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
      for (int v = 0; v < 4; ++v) Qj[v] = JQe[v * NG + p];
#pragma unroll
      for (int f = 0; f < 12; ++f) {
        gr[f] = GR[f * NG + p];
        lgr[f] = 0.0;
      }
      vort_vjp(Qj, jac[p], gr, A.eps_w, lq4, lgr);
#pragma unroll
      for (int f = 0; f < 12; ++f) LGR[f * NG + p] += lgr[f];
    }
    __syncthreads();
  }
  PHASE_MARK(23);

  // ---- reverse of pass 2: fluxes and interior divergence, grid by grid
  auto flux_dir = [&](auto Dc) {
    constexpr int D = decltype(Dc)::value;
    constexpr int xs = D == 0 ? 1 : (D == 1 ? G : G2);
    // LB, LL and LG hold grid D's points.  The lines of grid 0 are contiguous
    // runs of L doubles; when L is a power of two the 16 lines of a half-warp
    // would meet in two bank pairs, so point s of grid-0 line r is stored at
    // r*L + (s ^ ((r >> 1) & (L-1))) (a permutation within the line).
    auto sw = [](int i) -> int {
      if constexpr (D == 0 && (L & (L - 1)) == 0) return i ^ (((i / L) >> 1) & (L - 1));
      else return i;
    };
    // line phase: per line of grid D, the Lobatto state (LB), the 11 gradient
    // fields interpolated to the Lobatto points (into LG) and the transposed
    // derivative of dJ/dQt at the interior points (into LL), so that the point
    // phase reads each operand once
    for (int t = tid; t < 21 * G2; t += NT) {
      const int j = t / G2, ln = t - j * G2, a = ln % G, b = ln / G;
      const int p0 = gbase<G>(D, a, b), l0 = lbase<G>(D, a, b);
      double x[G];
      if (j < 5) {  // state field j
#pragma unroll
        for (int kk = 0; kk < G; ++kk) x[kk] = q[j * NG + p0 + kk * xs];
        LB[j * NL + sw(l0)] = QF[(face_lo(D) - 1) * 5 * G2 + j * G2 + ln];
        LB[j * NL + sw(l0 + (L - 1) * xs)] = QF[(face_hi(D) - 1) * 5 * G2 + j * G2 + ln];
#pragma unroll
        for (int s = 1; s < L - 1; ++s) {
          double acc = Op<G>::B(s, 0) * x[0];
#pragma unroll
          for (int kk = 1; kk < G; ++kk) acc = __fma_rn(Op<G>::B(s, kk), x[kk], acc);
          LB[j * NL + sw(l0 + s * xs)] = acc;
        }
      } else if (j < 16) {  // gradient field j-5 of grid D
        const int fi = diag_field(D, j - 5);
#pragma unroll
        for (int kk = 0; kk < G; ++kk) x[kk] = GR[fi * NG + p0 + kk * xs];
#pragma unroll
        for (int s = 0; s < L; ++s) {
          double acc = Op<G>::B(s, 0) * x[0];
#pragma unroll
          for (int kk = 1; kk < G; ++kk) acc = __fma_rn(Op<G>::B(s, kk), x[kk], acc);
          LG[(j - 5) * NL + sw(l0 + s * xs)] = acc;
        }
      } else {  // dJ/dQt of field j-16: -D^T along the line, interior points
        const int v = j - 16;
#pragma unroll
        for (int kk = 0; kk < G; ++kk) x[kk] = LAM[v * NG + p0 + kk * xs];
#pragma unroll
        for (int s = 1; s < L - 1; ++s) {
          double acc = 0.0;
#pragma unroll
          for (int kk = 0; kk < G; ++kk) acc += Op<G>::D(kk, s) * x[kk];
          LL[v * NL + sw(l0 + s * xs)] = -acc;
        }
      }
    }
    __syncthreads();
    PHASE_MARK(26);
    for (int qi = tid; qi < NL; qi += NT) {
      int s, a, b;
      ldecode<G>(D, qi, s, a, b);
      const int qs = sw(qi);
      double Q[NV], Gr[3][NV], lG[3][NV], lQ[NV], lfv[NV], fv[NV];
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        Q[v] = LB[v * NL + qs];
        lQ[v] = 0.0;
#pragma unroll
        for (int j = 0; j < 3; ++j) {
          Gr[j][v] = 0.0;
          lG[j][v] = 0.0;
        }
      }
#pragma unroll
      for (int jf = 0; jf < 11; ++jf) {
        const int fi = diag_field(D, jf);
        Gr[fi % 3][fi / 3] = LG[jf * NL + qs];
      }
      const double gd = gm[D * NL + qi];
      // entropy viscosity at this Lobatto point (EV_Prolong, as k_vol_diag): amu = 1 + mu
      // or Smagorinsky (nut_prolong, clipped at 0, as k_vol_diag): amu = 1 + nu rho
      constexpr bool ev = EVK;
      double amu = 1.0, lam = 0.0;
      [[maybe_unused]] double nuL = 0.0;
      [[maybe_unused]] bool nu_on = false;
      if constexpr (ev) {
        const int g0 = gbase<G>(D, a, b);
        double acc = Op<G>::B(s, 0) * MU[g0];
#pragma unroll
        for (int kk = 1; kk < G; ++kk) acc = __fma_rn(Op<G>::B(s, kk), MU[g0 + kk * xs], acc);
        if (A.les) {
          nu_on = !(acc < 0.0);
          nuL = nu_on ? acc : 0.0;
          amu = amu + nuL * Q[0];
        } else {
          amu = 1.0 + acc;
        }
      }
      double *lamp = ev ? &lam : nullptr;
      if (s == 0 || s == L - 1) {  // face point: VF = gd * fv
        const int fc = s == 0 ? face_lo(D) : face_hi(D);
        double lvf[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) {
          lvf[v] = LVF[(fc - 1) * 5 * G2 + v * G2 + a + G * b];
          lfv[v] = gd * lvf[v];
        }
        if (D == 0) vis_vjp<0>(Q, Gr, amu, P, lfv, fv, lQ, lG, lamp);
        else if (D == 1) vis_vjp<1>(Q, Gr, amu, P, lfv, fv, lQ, lG, lamp);
        else vis_vjp<2>(Q, Gr, amu, P, lfv, fv, lQ, lG, lamp);
#pragma unroll
        for (int v = 0; v < NV; ++v) lr += P.re * lvf[v] * (gd * fv[v]);
      } else {  // interior: F = gd fe - gd fv / Re, QTI += Dm F, Qt = -(QTI + ...)
        double lF[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) {
          lF[v] = LL[v * NL + qs];
          lfv[v] = -gd * P.r_re * lF[v];
        }
        double lfe[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) lfe[v] = gd * lF[v];
        if (D == 0) {
          vis_vjp<0>(Q, Gr, amu, P, lfv, fv, lQ, lG, lamp);
          euler_vjp<0>(Q, gamma, lfe, lQ);
        } else if (D == 1) {
          vis_vjp<1>(Q, Gr, amu, P, lfv, fv, lQ, lG, lamp);
          euler_vjp<1>(Q, gamma, lfe, lQ);
        } else {
          vis_vjp<2>(Q, Gr, amu, P, lfv, fv, lQ, lG, lamp);
          euler_vjp<2>(Q, gamma, lfe, lQ);
        }
#pragma unroll
        for (int v = 0; v < NV; ++v) lr += -gd * fv[v] * lF[v];
      }
#pragma unroll
      for (int v = 0; v < NV; ++v) LL[v * NL + qs] = lQ[v];
#pragma unroll
      for (int jf = 0; jf < 11; ++jf) {
        const int fi = diag_field(D, jf);
        LG[jf * NL + qs] = lG[fi % 3][fi / 3];
      }
      if constexpr (ev) {  // dJ/d(prolonged viscosity), in this point's (read) slot of field 0
        if (A.les) {
          LL[qs] += lam * nuL;  // amu = 1 + nu rho: the density's share
          LB[qs] = nu_on ? lam * Q[0] : 0.0;
        } else {
          LB[qs] = lam;
        }
      }
    }
    __syncthreads();
    PHASE_MARK(27);
    // transposed interpolations along the lines of D (and, with EV, of dJ/d amu
    // back to the Gauss-point viscosity)
    constexpr int ntr = EVK ? 17 * G2 : 16 * G2;
    for (int t = tid; t < ntr; t += NT) {
      const int j = t / G2, ln = t - j * G2, a = ln % G, b = ln / G;
      const int p0 = gbase<G>(D, a, b), l0 = lbase<G>(D, a, b);
      if (j < 11) {  // gradient field j of grid D -> its Gauss line
        const int fi = diag_field(D, j);
        double y[L];
#pragma unroll
        for (int s = 0; s < L; ++s) y[s] = LG[j * NL + sw(l0 + s * xs)];
#pragma unroll
        for (int kk = 0; kk < G; ++kk) {
          double acc = 0.0;
#pragma unroll
          for (int s = 0; s < L; ++s) acc += Op<G>::B(s, kk) * y[s];
          LGR[fi * NG + p0 + kk * xs] += acc;
        }
      } else if (j == 16) {  // EV_Prolong transposed
        double y[L];
#pragma unroll
        for (int s = 0; s < L; ++s) y[s] = LB[sw(l0 + s * xs)];
#pragma unroll
        for (int kk = 0; kk < G; ++kk) {
          double acc = 0.0;
#pragma unroll
          for (int s = 0; s < L; ++s) acc += Op<G>::B(s, kk) * y[s];
          LMU[p0 + kk * xs] += acc;
        }
      } else {  // state field v: interior Lobatto points -> q, end points -> QF
        const int v = j - 11;
        double y[L];
#pragma unroll
        for (int s = 0; s < L; ++s) y[s] = LL[v * NL + sw(l0 + s * xs)];
#pragma unroll
        for (int kk = 0; kk < G; ++kk) {
          double acc = 0.0;
#pragma unroll
          for (int s = 1; s < L - 1; ++s) acc += Op<G>::B(s, kk) * y[s];
          LQ[v * NG + p0 + kk * xs] += acc;
        }
        LQFs[(face_lo(D) - 1) * 5 * G2 + v * G2 + ln] += y[0];
        LQFs[(face_hi(D) - 1) * 5 * G2 + v * G2 + ln] += y[L - 1];
      }
    }
    __syncthreads();
  };
  flux_dir(std::integral_constant<int, 0>{});
  flux_dir(std::integral_constant<int, 1>{});
  flux_dir(std::integral_constant<int, 2>{});
  PHASE_MARK(24);

  // ---- reverse of pass 1: gradients -> Lobatto arrays -> q and QF
  auto lob_dir = [&](auto Dc) {
    constexpr int D = decltype(Dc)::value;
    constexpr int xs = D == 0 ? 1 : (D == 1 ? G : G2);
    for (int t = tid; t < 5 * G2; t += NT) {
      const int f = t / G2, ln = t - f * G2, a = ln % G, b = ln / G;
      const int p0 = gbase<G>(D, a, b);
      double lg[G];
#pragma unroll
      for (int kk = 0; kk < G; ++kk) lg[kk] = gg[D * NG + p0 + kk * xs] * LGR[(f * 3 + D) * NG + p0 + kk * xs];
      double y[L];
#pragma unroll
      for (int s = 0; s < L; ++s) {
        double acc = 0.0;
#pragma unroll
        for (int kk = 0; kk < G; ++kk) acc += Op<G>::D(kk, s) * lg[kk];
        y[s] = acc;
      }
#pragma unroll
      for (int kk = 0; kk < G; ++kk) {
        double acc = 0.0;
#pragma unroll
        for (int s = 1; s < L - 1; ++s) acc += Op<G>::B(s, kk) * y[s];
        LQ[f * NG + p0 + kk * xs] += acc;
      }
      LQFs[(face_lo(D) - 1) * 5 * G2 + f * G2 + ln] += y[0];
      LQFs[(face_hi(D) - 1) * 5 * G2 + f * G2 + ln] += y[L - 1];
    }
    __syncthreads();
  };
  lob_dir(std::integral_constant<int, 0>{});
  lob_dir(std::integral_constant<int, 1>{});
  lob_dir(std::integral_constant<int, 2>{});
  PHASE_MARK(25);

  // ---- reverse of the temperature gradients this stage saved for the next
  // step's entropy viscosity (vol_diag_tgrad): T1_D = gmetg(D,D) D T(Lobatto
  // line of the state along D), T = gamma p / rho (RHS.f90:66-83)
  if (EVK && !A.les && A.levb) {
    const double *lt1 = A.levb + (long long)k * 15 * NG + 12 * NG;
    auto tgrad_dir = [&](auto Dc) {
      constexpr int D = decltype(Dc)::value;
      constexpr int xs = D == 0 ? 1 : (D == 1 ? G : G2);
      for (int ln = tid; ln < G2; ln += NT) {
        const int a = ln % G, b = ln / G;
        const int p0 = gbase<G>(D, a, b);
        double y[NV][L];
#pragma unroll
        for (int v = 0; v < NV; ++v) {
          double x[G];
#pragma unroll
          for (int kk = 0; kk < G; ++kk) x[kk] = q[v * NG + p0 + kk * xs];
          y[v][0] = QF[(face_lo(D) - 1) * 5 * G2 + v * G2 + ln];
          y[v][L - 1] = QF[(face_hi(D) - 1) * 5 * G2 + v * G2 + ln];
#pragma unroll
          for (int s = 1; s < L - 1; ++s) {
            double acc = Op<G>::B(s, 0) * x[0];
#pragma unroll
            for (int kk = 1; kk < G; ++kk) acc = __fma_rn(Op<G>::B(s, kk), x[kk], acc);
            y[v][s] = acc;
          }
        }
        double ltd[G];
#pragma unroll
        for (int kk = 0; kk < G; ++kk) ltd[kk] = gg[D * NG + p0 + kk * xs] * lt1[D * NG + p0 + kk * xs];
        const double g = P.gamma, g1 = P.gamma - 1.0;
        const int l0 = lbase<G>(D, a, b);
#pragma unroll
        for (int s = 0; s < L; ++s) {  // dJ/d(Lobatto state) of T at each point, into LB
          double lT = 0.0;
#pragma unroll
          for (int kk = 0; kk < G; ++kk) lT += Op<G>::D(kk, s) * ltd[kk];
          const double rho = y[0][s], ri = 1.0 / rho;
          const double m2 = y[1][s] * y[1][s] + y[2][s] * y[2][s] + y[3][s] * y[3][s];
          const double p = g1 * (y[4][s] - 0.5 * m2 * ri);
          // T = g p / rho, p = (g - 1) (rho E - |m|^2 / (2 rho))
          LB[0 * NL + l0 + s * xs] = (g * g1 * 0.5 * m2 * ri * ri * ri - g * p * ri * ri) * lT;
#pragma unroll
          for (int i = 1; i <= 3; ++i) LB[i * NL + l0 + s * xs] = -g * g1 * y[i][s] * ri * ri * lT;
          LB[4 * NL + l0 + s * xs] = g * g1 * ri * lT;
        }
      }
      __syncthreads();
      for (int t = tid; t < 5 * G2; t += NT) {  // transposed interpolation: interior -> q, ends -> QF
        const int v = t / G2, ln = t - v * G2, a = ln % G, b = ln / G;
        const int p0 = gbase<G>(D, a, b), l0 = lbase<G>(D, a, b);
        double y[L];
#pragma unroll
        for (int s = 0; s < L; ++s) y[s] = LB[v * NL + l0 + s * xs];
#pragma unroll
        for (int kk = 0; kk < G; ++kk) {
          double acc = 0.0;
#pragma unroll
          for (int s = 1; s < L - 1; ++s) acc += Op<G>::B(s, kk) * y[s];
          LQ[v * NG + p0 + kk * xs] += acc;
        }
        LQFs[(face_lo(D) - 1) * 5 * G2 + v * G2 + ln] += y[0];
        LQFs[(face_hi(D) - 1) * 5 * G2 + v * G2 + ln] += y[L - 1];
      }
      __syncthreads();
    };
    tgrad_dir(std::integral_constant<int, 0>{});
    tgrad_dir(std::integral_constant<int, 1>{});
    tgrad_dir(std::integral_constant<int, 2>{});
  }

  // ---- outputs (the Jacobian's loads all in flight at once)
  {
    constexpr int NQ = (5 * NG + NT - 1) / NT;
    double jv[NQ];
#pragma unroll
    for (int j = 0; j < NQ; ++j) {
      const int i = tid + j * NT;
      if (i < 5 * NG) jv[j] = jac[i % NG];
    }
#pragma unroll
    for (int j = 0; j < NQ; ++j) {
      const int i = tid + j * NT;
      if (i < 5 * NG) LJQ[i] = jv[j] * LQ[i];
    }
  }
  for (int i = tid; i < 30 * G2; i += NT) A.LQF[(long long)k * 30 * G2 + i] = LQFs[i];
  if constexpr (EVK)
    for (int i = tid; i < NG; i += NT) A.lmuhg[(long long)k * NG + i] += LMU[i];
  // dJ/d(1/Re) of the element: warp sums, then the warps' sums in order
  static_assert(NT % 32 == 0 && NT / 32 <= 32, "whole warps, at most 32");
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) lr += __shfl_xor_sync(0xffffffffu, lr, o);
  if ((tid & 31) == 0) red[tid >> 5] = lr;
  __syncthreads();
  if (tid == 0) {
    double t = red[0];
    for (int w = 1; w < NT / 32; ++w) t += red[w];
    A.lr[k] += t;
  }
  PHASE_MARK(28);
}

// Direct part of the enstrophy term of a window step (energydissipation.f90:19-78):
// d eps / d JQe at fixed gradients, from the gradients the forward sweep saved
// for the step's last stage (EVB, [elem][15][G^3], fields as GR), added into
// dJ/dQ of the step's end state: LQ += w dvort/dJQe (the energy entry adds 0).
template <int G>
__global__ void __launch_bounds__(128) k_eps_dir(const double *__restrict__ JQe, const double *__restrict__ jac,
                                                  const double *__restrict__ EVB, double w, double *__restrict__ LQ) {
  constexpr int NG = G * G * G;
  const int k = blockIdx.x;
  const double *Jk = JQe + (long long)k * 5 * NG;
  const double *E = EVB + (long long)k * 15 * NG;
  const double *jk = jac + (long long)k * NG;
  double *Lk = LQ + (long long)k * 5 * NG;
  for (int p = threadIdx.x; p < NG; p += blockDim.x) {
    double Qj[4], gr[12], lgr[12], lq4[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int v = 0; v < 4; ++v) Qj[v] = Jk[v * NG + p];
#pragma unroll
    for (int f = 0; f < 12; ++f) {
      gr[f] = E[f * NG + p];
      lgr[f] = 0.0;
    }
    vort_vjp(Qj, jk[p], gr, w, lq4, lgr);
#pragma unroll
    for (int v = 0; v < 4; ++v) Lk[v * NG + p] += lq4[v];
    Lk[4 * NG + p] += 0.0;
  }
}

// out[0] += sum of part[0..n) (one block, fixed order)
__global__ void k_sum_into(const double *__restrict__ part, int n, double *__restrict__ out) {
  __shared__ double red[256];
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += 256) s += part[i];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[0] += red[0];
}

}  // namespace dsem
