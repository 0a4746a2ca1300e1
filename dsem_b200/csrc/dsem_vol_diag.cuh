// dsem_vol_diag.cuh -- volume kernel for elements with diagonal metrics (the
// axis-aligned hex elements of DSEM's boxes), sized for two CTAs per SM.
//
// Same mathematics and the same floating-point evaluation order as k_vol
// (Int_fluxes, Vis_Fluxes, Gauss_Deriv, update_interior:
// fluxesH_newa.f90:221-355, Vis_Fluxes_new.f90:16-382, SolnDerivsc.f90:14-83,
// updatea.f90:100-113), organised to keep about 107 KB of shared memory per
// element at p = 8 so that two elements share an SM and hide each other's
// latencies and barriers:
//
//  pass 1  one task per (direction D, field, line): the Lobatto line is built,
//          differentiated and scaled by gmetg(D,D) in registers; the Gauss
//          gradients of rho, rho u, rho v, rho w go to shared memory
//          (12 fields).  The energy gradients are not stored: each is needed
//          on one grid only and is recomputed there from that grid's line.
//  pass 2  per direction (z, y, x): the Lobatto arrays of grid D (5 fields,
//          and the energy gradient along D interpolated to grid D); then one
//          thread per Lobatto point interpolates the 11 gradient fields it
//          needs along D, evaluates the viscous and inviscid fluxes and
//          overwrites its own state slot with the flux; then one thread per
//          Gauss point adds the interior divergence along D to the element's
//          QTI slot (its own earlier writes, read back from L2).
// Every value is produced by the same FMA chain (same coefficients, same
// order) as in k_vol, so the two kernels agree bit for bit.
#pragma once
#include "dsem_stage.cuh"

namespace dsem {

// Launch shapes of k_vol_diag: threads per element (NT), the elements an SM
// must hold at once (MINB, which sets the register budget), elements per block
// (EPB: a block advances EPB elements one after another) and the Lobatto points
// per flux task (PPT: 2, two points of a line sharing each gradient-line load, or
// 1).  Variant 0 is the default; the autotuner (dsem_autotune) times variants
// 1..4 against it for p = 4, 6, 8: 1 and 2 change the threads and register
// budget, 3 takes two elements per block, 4 the other points-per-task.  Every
// variant evaluates each value with the same FMA chain, so all give identical
// results.
#ifndef DSEM_VOL_DIAG_NT8
#define DSEM_VOL_DIAG_NT8 192  // 2 CTAs x 6 warps per SM leave 168 registers per thread: no spills at p = 8
#endif
template <int G, int VV> struct VolDiagShape {
  // p >= 7: 192 / 128 / 256 threads, two elements per SM (168 / 255 / 128 registers)
  // p = 5, 6: 96 / 64 / 128 threads, four elements per SM (168 / 255 / 128 registers)
  // p <= 4: 64 / 64 / 128 threads, eight / six / four elements per SM
  // variants 3 and 4: the threads and register budget of variant 0
  static constexpr int V = VV >= 3 ? 0 : VV;
  static constexpr int NT = G >= 8 ? (V == 0 ? DSEM_VOL_DIAG_NT8 : (V == 1 ? 128 : 256))
                                   : G >= 6 ? (V == 0 ? 96 : (V == 1 ? 64 : 128))
                                            : G >= 4 ? (V == 2 ? 128 : 64) : 32;
#ifdef DSEM_VOL_DIAG_MINB
  static constexpr int MINB = V == 0 ? DSEM_VOL_DIAG_MINB : (G >= 8 ? 2 : (G >= 6 ? 4 : (V == 1 ? 6 : 4)));
#else
  static constexpr int MINB = G >= 8 ? 2 : (G >= 6 ? 4 : (G >= 4 ? (V == 0 ? 8 : (V == 1 ? 6 : 4)) : 16));
#endif
  static constexpr int EPB = VV == 3 ? 2 : 1;
  // points per flux task: p = 8 (G = 9) two by default, lower orders one (measured: 12 % faster
  // at p = 6); variant 4 takes the other
  static constexpr int PPT_DEFAULT = G >= 8 ? 2 : 1;
  static constexpr int PPT = VV == 4 ? 3 - PPT_DEFAULT : PPT_DEFAULT;
};

template <int G, bool EV, int SAVE, int V = 0> struct VolDiagCfg {
  static constexpr int L = G + 1, G2 = G * G, NG = G * G * G, NL = L * G * G;
  static constexpr int NT = VolDiagShape<G, V>::NT;
  static constexpr int NPT = (NG + NT - 1) / NT;       // Gauss points per thread (divergence)
  static constexpr int MINB = VolDiagShape<G, V>::MINB;
  static constexpr int EPB = VolDiagShape<G, V>::EPB, PPT = VolDiagShape<G, V>::PPT;
  static constexpr int NGR = 12;                        // Gauss gradients of fields 0..3
  static constexpr int NWORK = (6 * NL > 5 * NG) ? 6 * NL : 5 * NG;  // state (pass 1) / Lobatto arrays (pass 2)
  static constexpr size_t SMEM = sizeof(double) * (size_t)(NGR * NG + NWORK + 2 * G * L);
};

// Chain of contract<>(): acc = M(i,K0) x_K0, acc = fma(M(i,k), x_k, acc), with
// the row of M in registers (m[k - K0]) and x strided in memory.
template <int N> __device__ __forceinline__ double chain(const double *m, const double *x, int xs) {
  double acc = m[0] * x[0];
#pragma unroll
  for (int k = 1; k < N; ++k) acc = __fma_rn(m[k], x[k * xs], acc);
  return acc;
}

// Pass 1 task: field v (0..3) on line ln of direction D.  The Lobatto line is
// built (build_task of k_vol), differentiated and scaled by gmetg(D,D)
// (deriv_task) into GR.
template <int G, int D>
__device__ __forceinline__ void vol_diag_grad(int v, int ln, const double *WK, const double *QF, const double *gg,
                                              double *GR) {
  constexpr int L = G + 1, G2 = G * G, NG = G * G * G;
  constexpr int xs = D == 0 ? 1 : (D == 1 ? G : G2);
  const int a = ln % G, b = ln / G;
  const int p0 = gbase<G>(D, a, b);
  double y[L];
  {
    double x[G];
#pragma unroll
    for (int kk = 0; kk < G; ++kk) x[kk] = WK[v * NG + p0 + kk * xs];
    y[0] = QF[(face_lo(D) - 1) * 5 * G2 + v * G2 + ln];
    y[L - 1] = QF[(face_hi(D) - 1) * 5 * G2 + v * G2 + ln];
#pragma unroll
    for (int s = 1; s < L - 1; ++s) {  // build_task: contract<G, false, 1, L - 1, 0, G>
      double acc = Op<G>::B(s, 0) * x[0];
#pragma unroll
      for (int kk = 1; kk < G; ++kk) acc = __fma_rn(Op<G>::B(s, kk), x[kk], acc);
      y[s] = acc;
    }
  }
#pragma unroll
  for (int kk = 0; kk < G; ++kk) {  // deriv_task: contract_reg<G, true, 0, G, 0, L>
    double acc = Op<G>::D(kk, 0) * y[0];
#pragma unroll
    for (int s = 1; s < L; ++s) acc = __fma_rn(Op<G>::D(kk, s), y[s], acc);
    GR[(v * 3 + D) * NG + p0 + kk * xs] = gg[D * NG + p0 + kk * xs] * acc;
  }
}

// Temperature gradient along D (EV runs, SAVE == 2): the five Lobatto lines,
// the temperature on them (RHS.f90:66-83), its derivative scaled by gmetg(D,D).
template <int G, int D>
__device__ __forceinline__ void vol_diag_tgrad(int ln, const double *WK, const double *QF, const double *gg,
                                               double *EVB, double gamma) {
  constexpr int L = G + 1, G2 = G * G, NG = G * G * G;
  constexpr int xs = D == 0 ? 1 : (D == 1 ? G : G2);
  const int a = ln % G, b = ln / G;
  const int p0 = gbase<G>(D, a, b);
  double y[5][L];
#pragma unroll
  for (int v = 0; v < 5; ++v) {
    double x[G];
#pragma unroll
    for (int kk = 0; kk < G; ++kk) x[kk] = WK[v * NG + p0 + kk * xs];
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
  double T[L];
#pragma unroll
  for (int s = 0; s < L; ++s) {
    const double q1 = y[0][s], q2 = y[1][s], q3 = y[2][s], q4 = y[3][s], q5 = y[4][s];
    const double r1 = 1.0 / q1, u = ddiv(q2, q1, r1), v = ddiv(q3, q1, r1), w = ddiv(q4, q1, r1);
    const double Pp = (gamma - 1.0) * (q5 - 0.5 * q1 * (u * u + v * v + w * w));
    T[s] = ddiv(Pp * gamma, q1, r1);
  }
#pragma unroll
  for (int kk = 0; kk < G; ++kk) {
    double acc = Op<G>::D(kk, 0) * T[0];
#pragma unroll
    for (int s = 1; s < L; ++s) acc = __fma_rn(Op<G>::D(kk, s), T[s], acc);
    EVB[(12 + D) * NG + p0 + kk * xs] = gg[D * NG + p0 + kk * xs] * acc;
  }
}

// Fluxes at Lobatto point qi = (s; a, b) of grid D from its 11 interpolated
// gradient fields c (diag_field order; c[4] = energy gradient along D): the
// viscous flux times gmet at face points goes to VF, the inviscid minus viscous
// flux over Re overwrites the point's state slot in LB.
template <int G, int D>
__device__ __forceinline__ void vol_diag_point(int qi, int s, int a, int b, const double *c, bool les, double nu,
                                               bool ev, double mu, const Phys &P, const double *gm, double *LB,
                                               double *VF) {
  constexpr int L = G + 1, G2 = G * G, NL = L * G * G;
  double Q[NV], Qx[NV], Qy[NV], Qz[NV], r[NV], fl[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) Q[v] = LB[v * NL + qi];
  double amu = 1.0;  // Vis_Fluxes_new.f90:123-125
  if (les) amu = amu + nu * Q[0];
  if (ev) amu = amu + mu;
  const double rr = 1.0 / Q[0];
  const double gdiag = gm[D * NL + qi];
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
  if (s == 0 || s == L - 1) {
    const int fc = s == 0 ? face_lo(D) : face_hi(D);
#pragma unroll
    for (int v = 0; v < NV; ++v) VF[(fc - 1) * 5 * G2 + v * G2 + a + G * b] = r[v];
  } else {
    double fi[NV];
    euler_flux(D, Q, rr, P.gamma, fi);
#pragma unroll
    for (int v = 0; v < NV; ++v) LB[v * NL + qi] = gdiag * fi[v] - ddiv(r[v], P.re, P.r_re);
  }
}

// Pass 2 along direction D: Lobatto arrays of grid D, fluxes at its points,
// interior divergence accumulated into acc (the thread's Gauss points).
template <int G, bool EV, int SAVE, int D, int V>
__device__ __forceinline__ void vol_diag_dir(const VolArgs &A, const Phys &P, const double *JQ, const double *jac,
                                             const double *QF, const double *gg, const double *gm, const double *muhg,
                                             const double *nuhg,
                                             const double *GR, double *LB, double *T4, const double *Bm,
                                             const double *Dm, double *VF, double *QTI, int tid, long long &t_ph_) {
  using C = VolDiagCfg<G, EV, SAVE, V>;
  constexpr int L = G + 1, G2 = G * G, NG = G * G * G, NL = L * G * G, NT = C::NT, NPT = C::NPT;
  const int xs = D == 0 ? 1 : (D == 1 ? G : G2);
  const int ls = xs;  // Lobatto-grid stride along D (lstride)
  // (a) Lobatto arrays of grid D; the energy gradient along D on grid D (round robin, the
  // field-4 tasks -- line build, derivative and interpolation of the energy gradient, the
  // longest -- first)
  auto a_task = [&](int v, int ln) {
    const int a = ln % G, b = ln / G;
    const int p0 = gbase<G>(D, a, b), l0 = lbase<G>(D, a, b);
    double x[G], y[L];
#pragma unroll
    for (int kk = 0; kk < G; ++kk) x[kk] = JQ[v * NG + p0 + kk * xs] * jac[p0 + kk * xs];
    y[0] = QF[(face_lo(D) - 1) * 5 * G2 + v * G2 + ln];
    y[L - 1] = QF[(face_hi(D) - 1) * 5 * G2 + v * G2 + ln];
#pragma unroll
    for (int s = 1; s < L - 1; ++s) {
      double c = Op<G>::B(s, 0) * x[0];
#pragma unroll
      for (int kk = 1; kk < G; ++kk) c = __fma_rn(Op<G>::B(s, kk), x[kk], c);
      y[s] = c;
    }
#pragma unroll
    for (int s = 0; s < L; ++s) LB[v * NL + l0 + s * ls] = y[s];
    if (v == 4) {
      // gradient at Gauss point kk (deriv_task), streamed into the chains of
      // its interpolation to grid D (contract<G, false, 0, L, 0, G>)
      double t4[L];
#pragma unroll
      for (int kk = 0; kk < G; ++kk) {
        double c = Op<G>::D(kk, 0) * y[0];
#pragma unroll
        for (int s = 1; s < L; ++s) c = __fma_rn(Op<G>::D(kk, s), y[s], c);
        const double gq = gg[D * NG + p0 + kk * xs] * c;
#pragma unroll
        for (int s = 0; s < L; ++s) t4[s] = kk == 0 ? Op<G>::B(s, 0) * gq : __fma_rn(Op<G>::B(s, kk), gq, t4[s]);
      }
#pragma unroll
      for (int s = 0; s < L; ++s) T4[l0 + s * ls] = t4[s];
    }
  };
  for (int t = tid; t < 5 * G2; t += NT) a_task(4 - t / G2, t % G2);
  __syncthreads();
  PHASE_MARK(2 + 3 * (2 - D));
  // (b) fluxes at the Lobatto points of grid D (Vis_Fluxes_new.f90:115-228, fluxesH_newa.f90:276-352),
  // two points (s, s + NH) of one line per task so that both share the gradient loads.
  // Whole rounds of tasks first; the tasks of a last, partial round are split into
  // single points over twice as many threads, so that no thread computes two points
  // more than another.
  constexpr int NH = (L + 1) / 2;
  constexpr int NTB = NH * G2, RB = NTB / NT, LEFTB = NTB - RB * NT;
  constexpr bool SPLITB = LEFTB > 0 && 2 * LEFTB <= NT;
  auto b_task = [&](int t) {
    const int h = t / G2, ln = t - h * G2, a = ln % G, b = ln / G;
    const int g0 = gbase<G>(D, a, b), l0 = lbase<G>(D, a, b);
    const int s0 = h, s1 = h + NH;
    const bool two = s1 < L;
    const int s1c = two ? s1 : s0;
    double br0[G], br1[G];
#pragma unroll
    for (int kk = 0; kk < G; ++kk) {
      br0[kk] = Bm[s0 * G + kk];
      br1[kk] = Bm[s1c * G + kk];
    }
    double c0[11], c1[11];
#pragma unroll
    for (int jf = 0; jf < 11; ++jf) {
      if (jf == 4) {
        c0[jf] = T4[l0 + s0 * ls];
        c1[jf] = T4[l0 + s1c * ls];
      } else {
        const double *x = GR + diag_field(D, jf) * NG + g0;
        double xv[G];
#pragma unroll
        for (int kk = 0; kk < G; ++kk) xv[kk] = x[kk * xs];
        double a0 = br0[0] * xv[0], a1 = br1[0] * xv[0];
#pragma unroll
        for (int kk = 1; kk < G; ++kk) {
          a0 = __fma_rn(br0[kk], xv[kk], a0);
          a1 = __fma_rn(br1[kk], xv[kk], a1);
        }
        c0[jf] = a0;
        c1[jf] = a1;
      }
    }
    double mu0 = 0.0, mu1 = 0.0, nu0 = 0.0, nu1 = 0.0;
    if (EV) {  // EV_Prolong (Prolong_gtol.f90:7-51)
      mu0 = chain<G>(br0, muhg + g0, xs);
      mu1 = chain<G>(br1, muhg + g0, xs);
    }
    const bool les = nuhg != nullptr;
    if (les) {  // nut_prolong (staticSmag.f90:206-261): negative values clipped to 0
      nu0 = chain<G>(br0, nuhg + g0, xs);
      nu1 = chain<G>(br1, nuhg + g0, xs);
      if (nu0 < 0.0) nu0 = 0.0;
      if (nu1 < 0.0) nu1 = 0.0;
    }
    vol_diag_point<G, D>(l0 + s0 * ls, s0, a, b, c0, les, nu0, EV, mu0, P, gm, LB, VF);
    if (two) vol_diag_point<G, D>(l0 + s1 * ls, s1, a, b, c1, les, nu1, EV, mu1, P, gm, LB, VF);
  };
  // one point of task t: s = h (which == 0) or h + NH, the same chains as b_task
  auto b_point = [&](int t, int which) {
    const int h = t / G2, ln = t - h * G2, a = ln % G, b = ln / G;
    const int s0 = which ? h + NH : h;
    if (s0 >= L) return;
    const int g0 = gbase<G>(D, a, b), l0 = lbase<G>(D, a, b);
    double br0[G];
#pragma unroll
    for (int kk = 0; kk < G; ++kk) br0[kk] = Bm[s0 * G + kk];
    double c0[11];
#pragma unroll
    for (int jf = 0; jf < 11; ++jf) c0[jf] = jf == 4 ? T4[l0 + s0 * ls] : chain<G>(br0, GR + diag_field(D, jf) * NG + g0, xs);
    double mu0 = 0.0, nu0 = 0.0;
    if (EV) mu0 = chain<G>(br0, muhg + g0, xs);
    const bool les = nuhg != nullptr;
    if (les) {
      nu0 = chain<G>(br0, nuhg + g0, xs);
      if (nu0 < 0.0) nu0 = 0.0;
    }
    vol_diag_point<G, D>(l0 + s0 * ls, s0, a, b, c0, les, nu0, EV, mu0, P, gm, LB, VF);
  };
  if constexpr (C::PPT == 1) {  // one point per task
    for (int u = tid; u < 2 * NTB; u += NT) b_point(u >> 1, u & 1);
  } else if constexpr (SPLITB) {
    for (int t = tid; t < RB * NT; t += NT) b_task(t);
    if (tid < 2 * LEFTB) b_point(RB * NT + (tid >> 1), tid & 1);
  } else {
    for (int t = tid; t < NTB; t += NT) b_task(t);
  }
  // (c) interior divergence along D at this thread's Gauss points (updatea.f90:100-113),
  // summed over the directions in z, y, x order through the element's QTI slot; the
  // thread's own partial sums of the earlier directions (its own writes of the previous
  // phase (c)) are loaded before the barrier, so that their latency overlaps the wait
  double prev[NPT][NV];
  if (D != 2) {
#pragma unroll
    for (int j = 0; j < NPT; ++j) {
      const int p = tid + j * NT;
#pragma unroll
      for (int v = 0; v < NV; ++v) prev[j][v] = p < NG ? QTI[v * NG + p] : 0.0;
    }
  }
  __syncthreads();
  PHASE_MARK(3 + 3 * (2 - D));
#pragma unroll
  for (int j = 0; j < NPT; ++j) {
    const int p = tid + j * NT;
    if (p < NG) {
      const int n = p % G, m = (p / G) % G, l = p / G2;
      const int kk = D == 0 ? n : (D == 1 ? m : l);
      const int a = D == 0 ? m : n, b = D == 2 ? m : l;
      const double *f = LB + lbase<G>(D, a, b);
      double dr[L - 2];
#pragma unroll
      for (int s = 1; s < L - 1; ++s) dr[s - 1] = Dm[kk * L + s];
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        const double S = chain<L - 2>(dr, f + v * NL + ls, ls);
        QTI[v * NG + p] = (D == 2) ? S : prev[j][v] + S;
      }
    }
  }
  __syncthreads();
  PHASE_MARK(4 + 3 * (2 - D));
}

// One element k of the volume kernel (its block's threads, shared memory sm).
template <int G, bool EV, int SAVE, int V>
__device__ __forceinline__ void vol_diag_element(const VolArgs &A, const int k, double *sm) {
  using C = VolDiagCfg<G, EV, SAVE, V>;
  constexpr int L = G + 1, G2 = G * G, NG = G * G * G, NL = L * G * G, NT = C::NT;
  double *GR = sm;                  // [12][NG] Gauss gradients, field f*3 + direction
  double *WK = GR + C::NGR * NG;    // pass 1: state q [5][NG]; pass 2: LB [5][NL] + T4 [NL]
  double *LB = WK;
  double *T4 = WK + 5 * NL;         // energy gradient along D on grid D
  double *Bm = WK + C::NWORK;       // bx [L][G]
  double *Dm = Bm + L * G;          // dmx [G][L]
  const int tid = threadIdx.x;
  const double *JQ = A.JQ + (long long)k * A.sq;
  const double *jac = A.jac + (long long)k * NG;
  const double *QF = A.QF + (long long)k * 30 * G2;
  double *VF = A.VF + (long long)k * 30 * G2;
  const double *gg = A.gg + (long long)k * 3 * NG;
  const double *gm = A.gm + (long long)k * 3 * NL;
  const double *muhg = EV ? A.muhg + (long long)k * NG : nullptr;
  const double *nuhg = A.nuhg ? A.nuhg + (long long)k * NG : nullptr;
  double *EVB = SAVE ? A.EVB + (long long)k * 15 * NG : nullptr;
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

  // the element's metrics, face states and viscosities, read from the phases below,
  // are requested into L2 now (one bulk prefetch per array)
  if (tid == 0) {
    prefetch_l2_bulk(gg, 3 * NG);
    prefetch_l2_bulk(gm, 3 * NL);
    prefetch_l2_bulk(QF, 30 * G2);
    if (EV) prefetch_l2_bulk(muhg, NG);
    if (nuhg) prefetch_l2_bulk(nuhg, NG);
  }
  // operators to shared memory (rows are read at per-thread indices)
  for (int i = tid; i < L * G; i += NT) {
    Bm[i] = Op<G>::B(i / G, i % G);
    Dm[i] = Op<G>::D(i / L, i % L);
  }
  // Q*jacob (fluxesH_newa.f90:262-272), all of a thread's loads in flight at once
  {
    constexpr int NQ = (5 * NG + NT - 1) / NT;
    double qv[NQ], jv[NQ];
#pragma unroll
    for (int j = 0; j < NQ; ++j) {
      const int i = tid + j * NT;
      if (i < 5 * NG) {
        qv[j] = JQ[i];
        jv[j] = jac[i % NG];
      }
    }
#pragma unroll
    for (int j = 0; j < NQ; ++j) {
      const int i = tid + j * NT;
      if (i < 5 * NG) WK[i] = qv[j] * jv[j];
    }
  }
  __syncthreads();
  PHASE_MARK(0);

  // ---- pass 1: Gauss gradients of fields 0..3, one task per (direction, field, line)
  for (int t = tid; t < 12 * G2; t += NT) {
    const int f = t / G2, ln = t - f * G2;  // f = direction * 4 + field
    if (f < 4)
      vol_diag_grad<G, 0>(f, ln, WK, QF, gg, GR);
    else if (f < 8)
      vol_diag_grad<G, 1>(f - 4, ln, WK, QF, gg, GR);
    else
      vol_diag_grad<G, 2>(f - 8, ln, WK, QF, gg, GR);
  }
  if (SAVE == 2) {
    for (int t = tid; t < 3 * G2; t += NT) {
      const int D = t / G2, ln = t - D * G2;
      if (D == 0)
        vol_diag_tgrad<G, 0>(ln, WK, QF, gg, EVB, gamma);
      else if (D == 1)
        vol_diag_tgrad<G, 1>(ln, WK, QF, gg, EVB, gamma);
      else
        vol_diag_tgrad<G, 2>(ln, WK, QF, gg, EVB, gamma);
    }
  }
  __syncthreads();
  PHASE_MARK(1);
  if (SAVE) {
    for (int i = tid; i < 12 * NG; i += NT) EVB[i] = GR[i];
  }

  // ---- pass 2: z, y, x
  double *QTI = A.QTI + (long long)k * 5 * NG;
  vol_diag_dir<G, EV, SAVE, 2, V>(A, P, JQ, jac, QF, gg, gm, muhg, nuhg, GR, LB, T4, Bm, Dm, VF, QTI, tid, t_ph_);
  vol_diag_dir<G, EV, SAVE, 1, V>(A, P, JQ, jac, QF, gg, gm, muhg, nuhg, GR, LB, T4, Bm, Dm, VF, QTI, tid, t_ph_);
  vol_diag_dir<G, EV, SAVE, 0, V>(A, P, JQ, jac, QF, gg, gm, muhg, nuhg, GR, LB, T4, Bm, Dm, VF, QTI, tid, t_ph_);
  PHASE_MARK(20);
}

template <int G, bool EV, int SAVE, int V = 0>
__global__ void __launch_bounds__(VolDiagCfg<G, EV, SAVE, V>::NT, VolDiagCfg<G, EV, SAVE, V>::MINB)
    k_vol_diag(VolArgs A) {
  using C = VolDiagCfg<G, EV, SAVE, V>;
  extern __shared__ double sm[];
  if constexpr (C::EPB == 1) {
    vol_diag_element<G, EV, SAVE, V>(A, blockIdx.x, sm);
  } else {  // the block's elements one after another (each ends with a block barrier)
#pragma unroll 1
    for (int e = 0; e < C::EPB; ++e) {
      const int k = blockIdx.x * C::EPB + e;
      if (k >= A.nel) break;
      vol_diag_element<G, EV, SAVE, V>(A, k, sm);
    }
  }
}

}  // namespace dsem
