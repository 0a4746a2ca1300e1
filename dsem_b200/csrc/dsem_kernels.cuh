// dsem_kernels.cuh -- sm_100a FP64 kernels for DSEM's semi-discrete RHS and
// 2N-storage Runge-Kutta stage.
//
// Data layout in HBM (per order group; elements of one order are contiguous):
//   state  JQ, gQ, Qt_int : [elem][var][n + G*(m + G*l)]         (Gauss points)
//   faces  QF, FF, VF     : [elem][face 1..6][var][i + G*j]       (face-local index)
//   DIAG metrics          : jac [elem][G^3], gg [elem][3][G^3] (gmetg(d,d)),
//                           gm [elem][3][L*G^2] (gmet(d,d) on staggered grid d)
//   GENERAL metrics       : jac [elem][G^3], gg [elem][G^3][9] (gmetg(i,j), i+3j),
//                           gm [elem][3][L*G^2][3] (row d of gmet on grid d)
// Staggered grid d has L Lobatto points along d and G Gauss points in the
// other directions: grid 0 (lgg) n + L*(m + G*l), grid 1 (glg) n + G*(m + L*l),
// grid 2 (ggl) n + G*(m + G*l).
//
// Evaluation order is the oracle's (oracle/dsem_oracle.cpp): contractions are
// FMA chains in increasing summation index (explicit __fma_rn), pointwise
// physics is compiled without contraction (--fmad=false) in DSEM's expression
// order, and the divergence adds interior terms before the six face terms.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace dsem {

constexpr int NV = 5;
constexpr int GMIN = 2;
constexpr int GMAX = 9;  // p <= 8: one element's working set fits one CTA's shared memory

__host__ __device__ constexpr int ops_off(int G) {
  int o = 0;
  for (int g = GMIN; g < G; ++g) o += 2 * g * (g + 1);
  return o;
}
constexpr int OPS_TOTAL = ops_off(GMAX + 1);

// dmx [G][L] then bx [L][G] for every order G in [GMIN, GMAX]
static __constant__ double c_ops[OPS_TOTAL];  // one copy per translation unit, filled by Launch<G>::set_ops

template <int G> struct Op {
  static constexpr int L = G + 1;
  static constexpr int G2 = G * G;
  static constexpr int NG = G * G * G;
  static constexpr int NL = L * G * G;
  static constexpr int OD = ops_off(G);
  static constexpr int OB = ops_off(G) + G * (G + 1);
  __device__ __forceinline__ static double D(int k, int n) { return c_ops[OD + k * L + n]; }
  __device__ __forceinline__ static double B(int n, int j) { return c_ops[OB + n * G + j]; }
};

struct Phys {
  double gamma, re, pr, mach, cmu, mumax;
  int ducros;
  // correctly rounded reciprocals of the constant divisors, filled on the host
  double r_gm1, r_3, r_den, r_re;  // 1/(gamma-1), 1/3, 1/(pr*mach*mach*(gamma-1)), 1/re
};

// Fills the reciprocals of Phys from its constants (host side, IEEE division).
inline void phys_recips(Phys &P) {
  P.r_gm1 = 1.0 / (P.gamma - 1.0);
  P.r_3 = 1.0 / 3.0;
  P.r_den = 1.0 / (P.pr * P.mach * P.mach * (P.gamma - 1.0));
  P.r_re = 1.0 / P.re;
}

// Correctly rounded a/b from rb = RN(1/b): one Newton correction on the
// product, q = q0 + (a - b q0) rb with the residual exact through an FMA
// (P. Markstein, "Computation of elementary functions on the IBM RISC
// System/6000 processor", IBM J. Res. Develop. 34(1), 1990).  Equal to the
// IEEE quotient for the operand ranges of this solver (no overflow or
// underflow); the parity tests compare against plain division bit for bit.
__device__ __forceinline__ double ddiv(double a, double b, double rb) {
  const double q0 = a * rb;
  const double r = __fma_rn(-q0, b, a);
  return __fma_rn(r, rb, q0);
}

// Issues L2 prefetches for the n doubles at p, one 128-byte line per thread.
__device__ __forceinline__ void prefetch_l2(const double *p, int n, int tid, int nt) {
  const char *b = reinterpret_cast<const char *>(p);
  const long long lines = ((long long)n * 8 + 127) / 128;
  for (long long i = tid; i < lines; i += nt) {
    const char *a = b + i * 128;
    if (a >= b + (long long)n * 8) a = b + (long long)n * 8 - 8;  // stay inside the range
    asm volatile("prefetch.global.L2 [%0];" ::"l"(a));
  }
}

// One bulk L2 prefetch (cp.async.bulk.prefetch, a single instruction) of the
// n doubles at p.  The range is shrunk to whole 16-byte chunks inside
// [p, p + n): the start is rounded up and the end down, so nothing outside the
// array is touched; at most 8 bytes at either end are not prefetched.
__device__ __forceinline__ void prefetch_l2_bulk(const double *p, int n) {
  const unsigned long long a = reinterpret_cast<unsigned long long>(p);
  const unsigned long long lo = (a + 15ULL) & ~15ULL, hi = (a + 8ULL * (unsigned long long)n) & ~15ULL;
  if (hi > lo)
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(lo), "r"((unsigned)(hi - lo)) : "memory");
}

// ------------------------------------------------------------ line helpers
// Line (a,b) of direction d.  Gauss arrays: base/stride; grid-d arrays: base/stride.
template <int G> __device__ __forceinline__ int gbase(int d, int a, int b) {
  return d == 0 ? G * (a + G * b) : (d == 1 ? a + G * G * b : a + G * b);
}
template <int G> __device__ __forceinline__ int gstride(int d) { return d == 0 ? 1 : (d == 1 ? G : G * G); }
template <int G> __device__ __forceinline__ int lbase(int d, int a, int b) {
  constexpr int L = G + 1;
  return d == 0 ? L * (a + G * b) : (d == 1 ? a + G * L * b : a + G * b);
}
template <int G> __device__ __forceinline__ int lstride(int d) { return d == 0 ? 1 : (d == 1 ? G : G * G); }
// faces at the low/high Lobatto ends of direction d (DSEM numbering 1..6)
__device__ __forceinline__ int face_lo(int d) { return d == 0 ? 6 : (d == 1 ? 1 : 3); }
__device__ __forceinline__ int face_hi(int d) { return d == 0 ? 4 : (d == 1 ? 2 : 5); }
// decode a grid-d point index into (coordinate along d, a, b)
template <int G> __device__ __forceinline__ void ldecode(int d, int p, int &s, int &a, int &b) {
  constexpr int L = G + 1;
  if (d == 0) {
    s = p % L;
    int r = p / L;
    a = r % G;
    b = r / G;
  } else if (d == 1) {
    a = p % G;
    int r = p / G;
    s = r % L;
    b = r / L;
  } else {
    a = p % G;
    int r = p / G;
    b = r % G;
    s = r / G;
  }
}

// y[i*ys] = sum_{k=K0}^{K1-1} M(i,k) x[k*xs] for i in [I0,I1); FMA chain.
// DER selects dmx (G x L) else bx (L x G).
template <int G, bool DER, int I0, int I1, int K0, int K1>
__device__ __forceinline__ void contract(const double *__restrict__ x, int xs, double *__restrict__ y, int ys) {
  double r[K1 - K0];
#pragma unroll
  for (int k = K0; k < K1; ++k) r[k - K0] = x[k * xs];
#pragma unroll
  for (int i = I0; i < I1; ++i) {
    double acc = (DER ? Op<G>::D(i, K0) : Op<G>::B(i, K0)) * r[0];
#pragma unroll
    for (int k = K0 + 1; k < K1; ++k) acc = __fma_rn(DER ? Op<G>::D(i, k) : Op<G>::B(i, k), r[k - K0], acc);
    y[i * ys] = acc;
  }
}
template <int G, bool DER, int I0, int I1, int K0, int K1>
__device__ __forceinline__ void contract_reg(const double *__restrict__ x, int xs, double *out) {
  double r[K1 - K0];
#pragma unroll
  for (int k = K0; k < K1; ++k) r[k - K0] = x[k * xs];
#pragma unroll
  for (int i = I0; i < I1; ++i) {
    double acc = (DER ? Op<G>::D(i, K0) : Op<G>::B(i, K0)) * r[0];
#pragma unroll
    for (int k = K0 + 1; k < K1; ++k) acc = __fma_rn(DER ? Op<G>::D(i, k) : Op<G>::B(i, k), r[k - K0], acc);
    out[i - I0] = acc;
  }
}

// -------------------------------------------------------------- physics
// Euler flux of direction d (PhysLib.f90:17-124)
__device__ __forceinline__ void euler_flux(int d, const double *Q, double rr, double gamma, double *f) {
  double rho = Q[0], rhou = Q[1], rhov = Q[2], rhow = Q[3], rhoe = Q[4];
  double u = ddiv(rhou, rho, rr), v = ddiv(rhov, rho, rr), w = ddiv(rhow, rho, rr);
  double p = (gamma - 1.0) * (rhoe - 0.5 * rho * (u * u + v * v + w * w));
  if (d == 0) {
    f[0] = rhou; f[1] = p + rhou * u; f[2] = rhou * v; f[3] = rhou * w; f[4] = u * (rhoe + p);
  } else if (d == 1) {
    f[0] = rhov; f[1] = rhou * v; f[2] = p + rhov * v; f[3] = rhow * v; f[4] = v * (rhoe + p);
  } else {
    f[0] = rhow; f[1] = rhou * w; f[2] = rhov * w; f[3] = p + rhow * w; f[4] = w * (rhoe + p);
  }
}
__device__ __forceinline__ void euler_fluxes3(const double *Q, double rr, double gamma, double *f, double *g, double *h) {
  double rho = Q[0], rhou = Q[1], rhov = Q[2], rhow = Q[3], rhoe = Q[4];
  double u = ddiv(rhou, rho, rr), v = ddiv(rhov, rho, rr), w = ddiv(rhow, rho, rr);
  double p = (gamma - 1.0) * (rhoe - 0.5 * rho * (u * u + v * v + w * w));
  f[0] = rhou; f[1] = p + rhou * u; f[2] = rhou * v; f[3] = rhou * w; f[4] = u * (rhoe + p);
  g[0] = rhov; g[1] = rhou * v; g[2] = p + rhov * v; g[3] = rhow * v; g[4] = v * (rhoe + p);
  h[0] = rhow; h[1] = rhou * w; h[2] = rhov * w; h[3] = p + rhow * w; h[4] = w * (rhoe + p);
}

// Roe flux with entropy fix (PhysLib.f90:231-320)
__device__ __forceinline__ void riemann(const double *nh, double ds, const double *Ql, const double *Qr, double gamma,
                                        double *flux) {
  double rho = Ql[0], rhou = Ql[1], rhov = Ql[2], rhow = Ql[3], rhoe = Ql[4];
  double rhon = Qr[0], rhoun = Qr[1], rhovn = Qr[2], rhown = Qr[3], rhoen = Qr[4];
  const double rl = 1.0 / rho, rn = 1.0 / rhon;  // divisions by the densities: ddiv (correctly rounded)
  double ul = ddiv(rhou, rho, rl), vl = ddiv(rhov, rho, rl), wl = ddiv(rhow, rho, rl);
  double pleft = (gamma - 1.0) * (rhoe - ddiv(0.5, rho, rl) * (rhou * rhou + rhov * rhov + rhow * rhow));
  double ur = ddiv(rhoun, rhon, rn), vr = ddiv(rhovn, rhon, rn), wr = ddiv(rhown, rhon, rn);
  double pright = (gamma - 1.0) * (rhoen - ddiv(0.5, rhon, rn) * (rhoun * rhoun + rhovn * rhovn + rhown * rhown));
  double ql = nh[0] * ul + nh[1] * vl + nh[2] * wl;
  double qr = nh[0] * ur + nh[1] * vr + nh[2] * wr;
  const double gg1 = gamma / (gamma - 1.0);
  double hl = 0.5 * (ul * ul + vl * vl + wl * wl) + ddiv(gg1 * pleft, rho, rl);
  double hr = 0.5 * (ur * ur + vr * vr + wr * wr) + ddiv(gg1 * pright, rhon, rn);
  double rtd = sqrt(rho * rhon);
  double betal = rho / (rho + rtd);
  double betar = 1.0 - betal;
  double utd = betal * ul + betar * ur;
  double vtd = betal * vl + betar * vr;
  double wtd = betal * wl + betar * wr;
  double htd = betal * hl + betar * hr;
  double atd2 = (gamma - 1.0) * (htd - 0.5 * (utd * utd + vtd * vtd + wtd * wtd));
  double atd = sqrt(atd2);
  double qtd = utd * nh[0] + vtd * nh[1] + wtd * nh[2];
  if (qtd >= 0.0) {
    double dw1 = 0.5 * ((pright - pleft) / atd2 - (qr - ql) * rtd / atd);
    double sp1 = qtd - atd;
    double sp1m = sp1 <= 0.0 ? sp1 : 0.0;
    double hd1m = ((gamma + 1.0) / 4.0 * atd / rtd) * dw1;
    double e1 = -fabs(sp1) - hd1m;
    double eta1 = e1 >= 0.0 ? e1 : 0.0;
    double udw1 = dw1 * (sp1m - 0.5 * eta1);
    double rql = rho * ql;
    flux[0] = ds * (rql + udw1);
    flux[1] = ds * (rql * ul + pleft * nh[0] + udw1 * (utd - atd * nh[0]));
    flux[2] = ds * (rql * vl + pleft * nh[1] + udw1 * (vtd - atd * nh[1]));
    flux[3] = ds * (rql * wl + pleft * nh[2] + udw1 * (wtd - atd * nh[2]));
    flux[4] = ds * (rql * hl + udw1 * (htd - qtd * atd));
  } else {
    double dw4 = 0.5 * ((pright - pleft) / atd2 + (qr - ql) * rtd / atd);
    double sp4 = qtd + atd;
    double sp4p = sp4 >= 0.0 ? sp4 : 0.0;
    double hd4 = ((gamma + 1.0) / 4.0 * atd / rtd) * dw4;
    double e4 = -fabs(sp4) + hd4;
    double eta4 = e4 >= 0.0 ? e4 : 0.0;
    double udw4 = dw4 * (sp4p + 0.5 * eta4);
    double rqr = rhon * qr;
    flux[0] = ds * (rqr - udw4);
    flux[1] = ds * (rqr * ur + pright * nh[0] - udw4 * (utd + atd * nh[0]));
    flux[2] = ds * (rqr * vr + pright * nh[1] - udw4 * (vtd + atd * nh[1]));
    flux[3] = ds * (rqr * wr + pright * nh[2] - udw4 * (wtd + atd * nh[2]));
    flux[4] = ds * (rqr * hr - udw4 * (htd + qtd * atd));
  }
}

// Viscous fluxes (PhysLib.f90:419-583).  GX/GY/GZ hold the gradient
// components of the five conserved variables (x, y, z derivatives).
// The directional versions compute only what their flux vector reads.
__device__ __forceinline__ void vis_flux_x(const double *Q, double rr, const double *Qx, const double *Qy,
                                           const double *Qz, double amu, const Phys &P, double *f) {
  const double gamma = P.gamma;
  double rho = Q[0], rhou = Q[1], rhov = Q[2], rhow = Q[3], rhoe = Q[4];
  double u = ddiv(rhou, rho, rr), v = ddiv(rhov, rho, rr), w = ddiv(rhow, rho, rr);
  double p = (gamma - 1.0) * (rhoe - 0.5 * rho * (u * u + v * v + w * w));
  double ux = ddiv(Qx[1] - u * Qx[0], rho, rr), uy = ddiv(Qy[1] - u * Qy[0], rho, rr), uz = ddiv(Qz[1] - u * Qz[0], rho, rr);
  double vx = ddiv(Qx[2] - v * Qx[0], rho, rr), vy = ddiv(Qy[2] - v * Qy[0], rho, rr);
  double wx = ddiv(Qx[3] - w * Qx[0], rho, rr), wz = ddiv(Qz[3] - w * Qz[0], rho, rr);
  double px = (gamma - 1.0) * (Qx[4] - 0.5 * Qx[0] * (u * u + v * v + w * w) - rho * (u * ux + v * vx + w * wx));
  double tx = ddiv((px - ddiv(p * Qx[0], rho, rr)) * P.mach * P.mach * gamma, rho, rr);
  double akappa = 1.0 + ddiv((amu - 1.0) * 2.0e-1, gamma - 1.0, P.r_gm1);
  double div = ux + vy + wz;
  double sxy = uy + vx, sxz = wx + uz;
  f[0] = 0.0;
  f[1] = 2.0 * amu * (ux - ddiv(div, 3.0, P.r_3));
  f[2] = amu * sxy;
  f[3] = amu * sxz;
  f[4] = u * f[1] + v * f[2] + w * f[3] + ddiv(akappa * tx, P.pr * P.mach * P.mach * (gamma - 1.0), P.r_den);
}
__device__ __forceinline__ void vis_flux_y(const double *Q, double rr, const double *Qx, const double *Qy,
                                           const double *Qz, double amu, const Phys &P, double *g) {
  const double gamma = P.gamma;
  double rho = Q[0], rhou = Q[1], rhov = Q[2], rhow = Q[3], rhoe = Q[4];
  double u = ddiv(rhou, rho, rr), v = ddiv(rhov, rho, rr), w = ddiv(rhow, rho, rr);
  double p = (gamma - 1.0) * (rhoe - 0.5 * rho * (u * u + v * v + w * w));
  double ux = ddiv(Qx[1] - u * Qx[0], rho, rr), uy = ddiv(Qy[1] - u * Qy[0], rho, rr);
  double vx = ddiv(Qx[2] - v * Qx[0], rho, rr), vy = ddiv(Qy[2] - v * Qy[0], rho, rr), vz = ddiv(Qz[2] - v * Qz[0], rho, rr);
  double wy = ddiv(Qy[3] - w * Qy[0], rho, rr), wz = ddiv(Qz[3] - w * Qz[0], rho, rr);
  double py = (gamma - 1.0) * (Qy[4] - 0.5 * Qy[0] * (u * u + v * v + w * w) - rho * (u * uy + v * vy + w * wy));
  double ty = ddiv((py - ddiv(p * Qy[0], rho, rr)) * P.mach * P.mach * gamma, rho, rr);
  double akappa = 1.0 + ddiv((amu - 1.0) * 2.0e-1, gamma - 1.0, P.r_gm1);
  double div = ux + vy + wz;
  double sxy = uy + vx, syz = wy + vz;
  g[0] = 0.0;
  g[1] = amu * sxy;
  g[2] = 2.0 * amu * (vy - ddiv(div, 3.0, P.r_3));
  g[3] = amu * syz;
  g[4] = v * g[2] + u * g[1] + w * g[3] + ddiv(akappa * ty, P.pr * P.mach * P.mach * (gamma - 1.0), P.r_den);
}
__device__ __forceinline__ void vis_flux_z(const double *Q, double rr, const double *Qx, const double *Qy,
                                           const double *Qz, double amu, const Phys &P, double *h) {
  const double gamma = P.gamma;
  double rho = Q[0], rhou = Q[1], rhov = Q[2], rhow = Q[3], rhoe = Q[4];
  double u = ddiv(rhou, rho, rr), v = ddiv(rhov, rho, rr), w = ddiv(rhow, rho, rr);
  double p = (gamma - 1.0) * (rhoe - 0.5 * rho * (u * u + v * v + w * w));
  double ux = ddiv(Qx[1] - u * Qx[0], rho, rr), uz = ddiv(Qz[1] - u * Qz[0], rho, rr);
  double vy = ddiv(Qy[2] - v * Qy[0], rho, rr), vz = ddiv(Qz[2] - v * Qz[0], rho, rr);
  double wx = ddiv(Qx[3] - w * Qx[0], rho, rr), wy = ddiv(Qy[3] - w * Qy[0], rho, rr), wz = ddiv(Qz[3] - w * Qz[0], rho, rr);
  double pz = (gamma - 1.0) * (Qz[4] - 0.5 * Qz[0] * (u * u + v * v + w * w) - rho * (u * uz + v * vz + w * wz));
  double tz = ddiv((pz - ddiv(p * Qz[0], rho, rr)) * P.mach * P.mach * gamma, rho, rr);
  double akappa = 1.0 + ddiv((amu - 1.0) * 2.0e-1, gamma - 1.0, P.r_gm1);
  double div = ux + vy + wz;
  double sxz = wx + uz, syz = wy + vz;
  h[0] = 0.0;
  h[1] = amu * sxz;
  h[2] = amu * syz;
  h[3] = 2.0 * amu * (wz - ddiv(div, 3.0, P.r_3));
  h[4] = v * h[2] + u * h[1] + w * h[3] + ddiv(akappa * tz, P.pr * P.mach * P.mach * (gamma - 1.0), P.r_den);
}

// EV residual (EV_routines/Main/RHS.f90:207-278): D = ((phi+gam)/T)/Re
__device__ __forceinline__ double ev_residual(const Phys &P, const double *Q, const double *Qx, const double *Qy,
                                              const double *Qz, const double *T1, double &ducros) {
  const double gamma = P.gamma;
  double rho = Q[0], rhou = Q[1], rhov = Q[2], rhow = Q[3], rhoe = Q[4];
  double u = rhou / rho, v = rhov / rho, w = rhow / rho;
  double p = (gamma - 1.0) * (rhoe - 0.5 * rho * (u * u + v * v + w * w));
  double Tt = p * gamma / rho;
  double ux = (Qx[1] - u * Qx[0]) / rho, uy = (Qy[1] - u * Qy[0]) / rho, uz = (Qz[1] - u * Qz[0]) / rho;
  double vx = (Qx[2] - v * Qx[0]) / rho, vy = (Qy[2] - v * Qy[0]) / rho, vz = (Qz[2] - v * Qz[0]) / rho;
  double wx = (Qx[3] - w * Qx[0]) / rho, wy = (Qy[3] - w * Qy[0]) / rho, wz = (Qz[3] - w * Qz[0]) / rho;
  double tx = T1[0], ty = T1[1], tz = T1[2];
  double phi = (2.0 * (ux * ux + vy * vy + wz * wz) +
                ((vx + uy) * (vx + uy) + (uz + wx) * (uz + wx) + (vz + wy) * (vz + wy)) -
                2.0 * ((ux + vy + wz) * (ux + vy + wz)) / 3.0);
  double gam = (tx * tx + ty * ty + tz * tz) / (Tt * (gamma - 1.0) * P.pr);
  double div = ux + vy + wz;
  double cur = sqrt((wy - vz) * (wy - vz) + (uz - wx) * (uz - wx) + (vx - uy) * (vx - uy));
  double r = div * div / (div * div + cur * cur + 1.0e-9);
  double mn = 1.0 <= r ? 1.0 : r;
  ducros = 0.0 >= mn ? 0.0 : mn;
  return (((phi + gam) / Tt) / P.re);
}

// Density-based sensor of calculate_terms (RHS.f90:264-275) from the density gradient
__device__ __forceinline__ double rho_sensor(double rx, double ry, double rz) {
  const double eps = 1.0e-9;
  const double rhoX2 = rx * rx, rhoY2 = ry * ry, rhoZ2 = rz * rz;
  return sqrt((1.0 / ((1.0 / (rhoX2 + eps)) + (1.0 / (rhoY2 + eps)) + 1.0)) +
              (1.0 / ((1.0 / (rhoX2 + eps)) + (1.0 / (rhoZ2 + eps)) + 1.0)) +
              (1.0 / ((1.0 / (rhoY2 + eps)) + (1.0 / (rhoZ2 + eps)) + 1.0)));
}

// gradient fields interpolated to grid d for the directional viscous flux
// (field id = var*3 + derivative direction)
__device__ __forceinline__ int diag_field(int d, int j) {
  // d=0: Qx[0..4], Qy[0,1,2], Qz[0,1,3]; d=1: Qy[0..4], Qx[0,1,2], Qz[0,2,3]; d=2: Qz[0..4], Qx[0,1,3], Qy[0,2,3]
  const int t0[11] = {0, 3, 6, 9, 12, 1, 4, 7, 2, 5, 11};
  const int t1[11] = {1, 4, 7, 10, 13, 0, 3, 6, 2, 8, 11};
  const int t2[11] = {2, 5, 8, 11, 14, 0, 3, 9, 1, 7, 10};
  return d == 0 ? t0[j] : (d == 1 ? t1[j] : t2[j]);
}

}  // namespace dsem
