// dsem_inst.cuh -- definitions of Launch<G>; included once per order by inst_g*.cu.
#pragma once
#include "dsem_launch.h"
#include "dsem_stage.cuh"
#include "dsem_vol_diag.cuh"
#include "dsem_lobatto.cuh"

namespace dsem {

template <int G> cudaError_t Launch<G>::set_ops(const double *h, int n) {
  if (n != OPS_TOTAL) return cudaErrorInvalidValue;
  return cudaMemcpyToSymbol(c_ops, h, sizeof(double) * OPS_TOTAL);
}

template <int G, bool DIAG, bool EV, int SAVE> static cudaError_t vol_one(const VolArgs &a, int nel, cudaStream_t s) {
  using C = VolCfg<G, DIAG, EV, SAVE>;
  auto kern = k_vol<G, DIAG, EV, SAVE>;
  static std::atomic<unsigned long long> attr{0};
  cudaError_t e = set_smem_once(kern, C::SMEM, attr);
  if (e != cudaSuccess) return e;
  if (nel <= 0) return cudaSuccess;
  kern<<<nel, C::NT, C::SMEM, s>>>(a);
  return cudaGetLastError();
}

// diagonal metrics: k_vol_diag (two elements per SM at p = 8)
template <int G, bool EV, int SAVE, int V = 0>
static cudaError_t vol_diag_one(const VolArgs &a, int nel, cudaStream_t s) {
  using C = VolDiagCfg<G, EV, SAVE, V>;
  auto kern = k_vol_diag<G, EV, SAVE, V>;
  static std::atomic<unsigned long long> attr{0};
  cudaError_t e = set_smem_once(kern, C::SMEM, attr);
  if (e != cudaSuccess) return e;
  if (nel <= 0) return cudaSuccess;
  VolArgs b = a;
  b.nel = nel;
  kern<<<(nel + C::EPB - 1) / C::EPB, C::NT, C::SMEM, s>>>(b);
  return cudaGetLastError();
}

template <int G> size_t Launch<G>::vol_smem(bool diag, int mode) {
  switch (mode) {
    case VOL_SAVE: return diag ? VolDiagCfg<G, false, 1>::SMEM : VolCfg<G, false, false, 1>::SMEM;
    case VOL_EV: return diag ? VolDiagCfg<G, true, 0>::SMEM : VolCfg<G, false, true, 0>::SMEM;
    case VOL_EV_SAVE: return diag ? VolDiagCfg<G, true, 2>::SMEM : VolCfg<G, false, true, 2>::SMEM;
    default: return diag ? VolDiagCfg<G, false, 0>::SMEM : VolCfg<G, false, false, 0>::SMEM;
  }
}
template <int G> int Launch<G>::vol_threads(bool diag, int mode) {
  (void)mode;
  return diag ? VolDiagCfg<G, false, 0>::NT : VolCfg<G, false, false, 0>::NT;
}

// launch-shape variants of k_vol_diag instantiated for this order (p = 4, 6, 8)
template <int G> int Launch<G>::vol_variants() { return (G == 5 || G == 7 || G == 9) ? VOL_VARIANTS : 1; }

template <int G> int Launch<G>::vol_variant_threads(int v) {
  switch (v) {
    case 1: return VolDiagShape<G, 1>::NT;
    case 2: return VolDiagShape<G, 2>::NT;
    case 3: return VolDiagShape<G, 3>::NT;
    case 4: return VolDiagShape<G, 4>::NT;
    default: return VolDiagShape<G, 0>::NT;
  }
}

template <int G>
cudaError_t Launch<G>::vol(const VolArgs &a, int nel, bool diag, int mode, cudaStream_t s, int variant) {
  if constexpr (G == 5 || G == 7 || G == 9) {  // variants of the diagonal kernel without entropy viscosity
    if (diag && variant >= 1 && variant < VOL_VARIANTS && (mode == VOL_PLAIN || mode == VOL_SAVE)) {
      const bool sv = mode == VOL_SAVE;
      switch (variant) {
        case 1: return sv ? vol_diag_one<G, false, 1, 1>(a, nel, s) : vol_diag_one<G, false, 0, 1>(a, nel, s);
        case 2: return sv ? vol_diag_one<G, false, 1, 2>(a, nel, s) : vol_diag_one<G, false, 0, 2>(a, nel, s);
        case 3: return sv ? vol_diag_one<G, false, 1, 3>(a, nel, s) : vol_diag_one<G, false, 0, 3>(a, nel, s);
        default: return sv ? vol_diag_one<G, false, 1, 4>(a, nel, s) : vol_diag_one<G, false, 0, 4>(a, nel, s);
      }
    }
  }
  switch (mode) {
    case VOL_SAVE: return diag ? vol_diag_one<G, false, 1>(a, nel, s) : vol_one<G, false, false, 1>(a, nel, s);
    case VOL_EV: return diag ? vol_diag_one<G, true, 0>(a, nel, s) : vol_one<G, false, true, 0>(a, nel, s);
    case VOL_EV_SAVE: return diag ? vol_diag_one<G, true, 2>(a, nel, s) : vol_one<G, false, true, 2>(a, nel, s);
    default: return diag ? vol_diag_one<G, false, 0>(a, nel, s) : vol_one<G, false, false, 0>(a, nel, s);
  }
}

template <int G> cudaError_t Launch<G>::update(const UpdArgs &a, int nel, cudaStream_t s) {
  if (nel <= 0) return cudaSuccess;
  const size_t smem = sizeof(double) * (30 * G * G + 5 * G * G * G + 2 * G);
  if (a.fmc)
    k_update<G, true><<<nel, 256, smem, s>>>(a);
  else
    k_update<G, false><<<nel, 256, smem, s>>>(a);
  return cudaGetLastError();
}

template <int G> cudaError_t Launch<G>::trace(const TraceArgs &a, int nel, cudaStream_t s) {
  if (nel <= 0) return cudaSuccess;
  k_trace<G><<<nel, 256, sizeof(double) * 5 * G * G * G, s>>>(a);
  return cudaGetLastError();
}

template <int G> cudaError_t Launch<G>::lob_keep(const LobArgs &a, int nel, cudaStream_t s) {
  if (nel <= 0) return cudaSuccess;
  k_lob_keep<G><<<nel, 256, sizeof(double) * 5 * G * G * G, s>>>(a);
  return cudaGetLastError();
}

template <int G> cudaError_t Launch<G>::lob_grad(const LobArgs &a, int nel, bool diag, cudaStream_t s) {
  if (nel <= 0) return cudaSuccess;
  if (diag)
    k_lob_grad<G, true><<<nel, 256, 0, s>>>(a);
  else
    k_lob_grad<G, false><<<nel, 256, 0, s>>>(a);
  return cudaGetLastError();
}

template <int G> cudaError_t Launch<G>::ev(const EvArgs &a, int nel, cudaStream_t s) {
  if (nel <= 0) return cudaSuccess;
  k_ev<G><<<nel, 256, 0, s>>>(a);
  return cudaGetLastError();
}

template <int G> cudaError_t Launch<G>::les(const LesArgs &a, int nel, cudaStream_t s) {
  if (nel <= 0) return cudaSuccess;
  k_les<G><<<nel, 128, 0, s>>>(a);
  return cudaGetLastError();
}

template <int G>
cudaError_t Launch<G>::face_inv(const MortarC *mc, int nm, double *QF, double *FF, const double *nh, const double *nrm,
                                double gamma, cudaStream_t s) {
  if (nm <= 0) return cudaSuccess;
  const long long n = (long long)nm * G * G;
  k_face_inv<G><<<(unsigned)((n + 127) / 128), 128, 0, s>>>(mc, nm, QF, FF, nh, nrm, gamma);
  return cudaGetLastError();
}

template <int G>
cudaError_t Launch<G>::face_inv_from(const MortarC *mc, int nm, const double *QFR, double *QF, double *FF,
                                     const double *nh, const double *nrm, double gamma, cudaStream_t s) {
  if (nm <= 0) return cudaSuccess;
  const long long n = (long long)nm * G * G;
  k_face_inv_from<G><<<(unsigned)((n + 127) / 128), 128, 0, s>>>(mc, nm, QFR, QF, FF, nh, nrm, gamma);
  return cudaGetLastError();
}

template <int G> cudaError_t Launch<G>::face_vis(const MortarC *mc, int nm, double *VF, const double *nrm, cudaStream_t s) {
  if (nm <= 0) return cudaSuccess;
  const long long n = (long long)nm * G * G;
  k_face_vis<G><<<(unsigned)((n + 127) / 128), 128, 0, s>>>(mc, nm, VF, nrm);
  return cudaGetLastError();
}

template <int G>
cudaError_t Launch<G>::face_inv_cut(const MortarCut *mc, int nm, double *QF, double *FF, const double *ghost,
                                    const double *nh, const double *nrm, double gamma, cudaStream_t s) {
  if (nm <= 0) return cudaSuccess;
  const long long n = (long long)nm * G * G;
  k_face_inv_cut<G><<<(unsigned)((n + 127) / 128), 128, 0, s>>>(mc, nm, QF, FF, ghost, nh, nrm, gamma);
  return cudaGetLastError();
}

template <int G>
cudaError_t Launch<G>::face_vis_cut(const MortarCut *mc, int nm, double *VF, const double *ghost, const double *nrm,
                                    cudaStream_t s) {
  if (nm <= 0) return cudaSuccess;
  const long long n = (long long)nm * G * G;
  k_face_vis_cut<G><<<(unsigned)((n + 127) / 128), 128, 0, s>>>(mc, nm, VF, ghost, nrm);
  return cudaGetLastError();
}

template <int G>
cudaError_t Launch<G>::face_bnd_inv(const MortarB *mb, int nm, double *QF, double *FF, const double *nh,
                                    const double *nrm, const double *qext, const BndPhys &P, cudaStream_t s) {
  if (nm <= 0) return cudaSuccess;
  const long long n = (long long)nm * G * G;
  k_face_bnd_inv<G><<<(unsigned)((n + 127) / 128), 128, 0, s>>>(mb, nm, QF, FF, nh, nrm, qext, P);
  return cudaGetLastError();
}

template <int G>
cudaError_t Launch<G>::face_bnd_vis(const MortarB *mb, int nm, double *VF, const double *nrm, const double *fvext,
                                    cudaStream_t s) {
  if (nm <= 0) return cudaSuccess;
  const long long n = (long long)nm * G * G;
  k_face_bnd_vis<G><<<(unsigned)((n + 127) / 128), 128, 0, s>>>(mb, nm, VF, nrm, fvext);
  return cudaGetLastError();
}

}  // namespace dsem

#define DSEM_INSTANTIATE(GG) template struct dsem::Launch<GG>;
