// dsem_lobatto.cuh -- the Lobatto arrays of the last stage (DSEM's d%Qlgg,
// d%Qglg, d%Qggl) kept in device memory, and the Gauss gradients rebuilt
// from them.
//
// DSEM's restart file stores the three Lobatto arrays of the last Fluxes call
// (write_restart, Parabolic3D/stac3m/restart.f90:116-118); its entropy
// viscosity and Smagorinsky model read them at the start of the next step
// (RHS_ent_trans, EV_routines/Main/RHS.f90:21-190).  The volume kernels keep
// only the gradients derived from them (EVB), so:
//   k_lob_keep   rebuilds, in the last stage, the Lobatto arrays the volume
//                kernel builds (interior points from Q*jacob, face points from
//                the averaged face state: the same FMA chains) and stores them,
//                [elem][grid d][5][L*G^2], grid d with L points along d;
//   k_lob_grad   turns stored arrays (from that kernel or from a restart file)
//                into the saved gradients EVB: Gauss gradients of rho, rho u,
//                rho v, rho w and of T, the same chains as the volume kernels'
//                pass 1 (Gauss_Deriv, SolnDerivsc.f90:36-80; T from RHS.f90:66-83).
#pragma once
#include "dsem_stage.cuh"

namespace dsem {

struct LobArgs {
  const double *JQ;
  long long sq;
  const double *jac, *gg;  // gg: diagonal [elem][3][G^3] or general [elem][G^3][9]
  const double *QF;        // averaged face state
  double *QLB;             // [elem][3][5][L*G^2]
  double *EVB;             // [elem][15][G^3]
  double gamma;
};

template <int G> __global__ void __launch_bounds__(256) k_lob_keep(LobArgs A) {
  constexpr int L = G + 1, G2 = G * G, NG = G * G * G, NL = L * G * G;
  extern __shared__ double q[];  // [5][NG]: Q*jacob (fluxesH_newa.f90:262-272)
  const int k = blockIdx.x, tid = threadIdx.x, nt = blockDim.x;
  const double *JQ = A.JQ + (long long)k * A.sq;
  const double *jac = A.jac + (long long)k * NG;
  const double *QF = A.QF + (long long)k * 30 * G2;
  double *out = A.QLB + (long long)k * 15 * NL;
  for (int i = tid; i < 5 * NG; i += nt) q[i] = JQ[i] * jac[i % NG];
  __syncthreads();
  for (int t = tid; t < 15 * G2; t += nt) {
    const int D = t / (5 * G2), r = t - D * 5 * G2;
    if (D == 0)
      build_task<G, L, 0>(r, q, QF, out, NL);
    else if (D == 1)
      build_task<G, L, 1>(r, q, QF, out + 5 * NL, NL);
    else
      build_task<G, L, 2>(r, q, QF, out + 10 * NL, NL);
  }
}

// One CTA per element; the directions in order 0, 1, 2 (the general metric sums
// the three contributions of each gradient in that order, as k_vol does).
template <int G, bool DIAG> __global__ void __launch_bounds__(256) k_lob_grad(LobArgs A) {
  constexpr int L = G + 1, G2 = G * G, NG = G * G * G, NL = L * G * G;
  const int k = blockIdx.x, tid = threadIdx.x, nt = blockDim.x;
  const double *lb = A.QLB + (long long)k * 15 * NL;
  const double *gg = A.gg + (long long)k * 3 * NG * (DIAG ? 1 : 3);
  double *EVB = A.EVB + (long long)k * 15 * NG;
  // fields 0..3 (rho, rho u, rho v, rho w) -> EVB[f*3 + c]; field "5" (T) -> EVB[12 + c]
  for (int t = tid; t < 5 * G2; t += nt) {
    const int f = t / G2, tt = (f < 4 ? f : 5) * G2 + (t - f * G2);
    deriv_task<G, L, DIAG, 0>(tt, lb, NL, gg, EVB, EVB, A.gamma);
  }
  __syncthreads();
  for (int t = tid; t < 5 * G2; t += nt) {
    const int f = t / G2, tt = (f < 4 ? f : 5) * G2 + (t - f * G2);
    deriv_task<G, L, DIAG, 1>(tt, lb + 5 * NL, NL, gg, EVB, EVB, A.gamma);
  }
  __syncthreads();
  for (int t = tid; t < 5 * G2; t += nt) {
    const int f = t / G2, tt = (f < 4 ? f : 5) * G2 + (t - f * G2);
    deriv_task<G, L, DIAG, 2>(tt, lb + 10 * NL, NL, gg, EVB, EVB, A.gamma);
  }
}

}  // namespace dsem
