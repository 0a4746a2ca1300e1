// dsem_launch.h -- host-side launch interface of the per-order kernel
// instantiations (one translation unit per order G = p+1, see inst_g*.cu).
#pragma once
#include <cuda_runtime.h>

#include <atomic>

namespace dsem {

struct Phys;
struct VolArgs;
struct UpdArgs;
struct TraceArgs;
struct EvArgs;
struct LesArgs;
struct MortarC;
struct MortarCut;
struct MortarB;
struct BndPhys;
struct LobArgs;

// A kernel's dynamic shared-memory limit is a per-device setting: raises it to
// smem on the current device the first time that device launches kern (mask:
// the call site's record of the devices done, one bit per device id < 64).
template <class K>
cudaError_t set_smem_once(K kern, size_t smem, std::atomic<unsigned long long> &mask) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const unsigned long long bit = (dev >= 0 && dev < 64) ? 1ULL << dev : 0ULL;
  if (bit && (mask.load(std::memory_order_relaxed) & bit)) return cudaSuccess;
  e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess && bit) mask.fetch_or(bit, std::memory_order_relaxed);
  return e;
}

// volume kernel variants: metric layout x entropy viscosity x saved gradients
enum VolMode { VOL_PLAIN = 0, VOL_SAVE = 1, VOL_EV = 2, VOL_EV_SAVE = 3 };
// launch shapes of the diagonal volume kernel the autotuner chooses from
constexpr int VOL_VARIANTS = 5;

template <int G> struct Launch {
  static cudaError_t set_ops(const double *host_ops, int n);  // copies the operator table to constant memory
  static size_t vol_smem(bool diag, int mode);
  static int vol_threads(bool diag, int mode);
  static cudaError_t vol(const VolArgs &a, int nel, bool diag, int mode, cudaStream_t s, int variant = 0);
  static int vol_variants();                // launch shapes available for this order (1 or VOL_VARIANTS)
  static int vol_variant_threads(int v);    // threads per element of shape v
  static cudaError_t update(const UpdArgs &a, int nel, cudaStream_t s);
  static cudaError_t trace(const TraceArgs &a, int nel, cudaStream_t s);
  // Lobatto arrays of the stage kept in a.QLB; gradients rebuilt from them into a.EVB
  static cudaError_t lob_keep(const LobArgs &a, int nel, cudaStream_t s);
  static cudaError_t lob_grad(const LobArgs &a, int nel, bool diag, cudaStream_t s);
  static cudaError_t ev(const EvArgs &a, int nel, cudaStream_t s);
  static cudaError_t les(const LesArgs &a, int nel, cudaStream_t s);
  static cudaError_t face_inv(const MortarC *mc, int nm, double *QF, double *FF, const double *nh, const double *nrm,
                              double gamma, cudaStream_t s);
  // the same from raw traces QFR kept elsewhere (left unchanged), averages into QF
  static cudaError_t face_inv_from(const MortarC *mc, int nm, const double *QFR, double *QF, double *FF,
                                   const double *nh, const double *nrm, double gamma, cudaStream_t s);
  static cudaError_t face_vis(const MortarC *mc, int nm, double *VF, const double *nrm, cudaStream_t s);
  static cudaError_t face_inv_cut(const MortarCut *mc, int nm, double *QF, double *FF, const double *ghost,
                                  const double *nh, const double *nrm, double gamma, cudaStream_t s);
  static cudaError_t face_vis_cut(const MortarCut *mc, int nm, double *VF, const double *ghost, const double *nrm,
                                  cudaStream_t s);
  static cudaError_t face_bnd_inv(const MortarB *mb, int nm, double *QF, double *FF, const double *nh,
                                  const double *nrm, const double *qext, const BndPhys &P, cudaStream_t s);
  static cudaError_t face_bnd_vis(const MortarB *mb, int nm, double *VF, const double *nrm, const double *fvext,
                                  cudaStream_t s);
};

}  // namespace dsem
