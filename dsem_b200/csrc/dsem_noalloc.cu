// dsem_noalloc.cu -- dsem_rhs_noalloc: the right-hand side of dsem_rhs for
// callers that cannot allocate device memory.
//
// Some host applications own all of the GPU's memory through their own pool
// allocator, or fix their device-memory budget when they start; a library
// that calls cudaMalloc behind their back fails or breaks that budget.  This
// entry point allocates nothing: the caller passes its inputs and outputs in
// device memory, and the working buffers of the pipeline (face traces, face
// fluxes, viscous face fluxes, interior divergence and an error flag) live in
// one file-scope static device array of DSEM_NOALLOC_SCRATCH_DOUBLES doubles
// (8 MiB), which every GPU that loads the library holds until the process
// exits.
//
// Contract (see include/dsem_gpu.h):
//  - the first call on a device does the per-device set-up (symbol address of
//    the scratch array, operator tables in constant memory, kernel
//    attributes), with that device current;
//  - no call may be made while its stream is being captured: every call
//    clears the scratch, reads its flag back and waits for the stream, so it
//    returns DSEM_ERR_INVALID_ARG on a capturing stream;
//  - every call shares the one scratch array and leaves its contents behind;
//    calls whose work overlaps on the GPU (two streams, two host threads)
//    race on it and must be serialised by the caller;
//  - the call enqueues on the caller's stream and waits for it before
//    returning.
#include <cuda_runtime.h>

#include <mutex>
#include <string>
#include <type_traits>

#include "../../include/dsem_gpu.h"
#include "dsem_host_math.h"
#include "dsem_launch.h"
#include "dsem_stage.cuh"

using namespace dsem;

void dsem_set_thread_error(const std::string &msg);  // dsem_api.cu

namespace {

static __device__ __align__(256) double g_noalloc_scratch[DSEM_NOALLOC_SCRATCH_DOUBLES];

constexpr int MAX_DEVICES = 64;
std::mutex g_setup_mutex;
double *g_scratch_ptr[MAX_DEVICES] = {};
int nfail(int code, const std::string &msg) {
  dsem_set_thread_error(msg);  // reported by dsem_last_error(NULL)
  return code;
}

template <class F> cudaError_t with_G(int G, F &&f) {
  switch (G) {
    case 2: return f(std::integral_constant<int, 2>{});
    case 3: return f(std::integral_constant<int, 3>{});
    case 4: return f(std::integral_constant<int, 4>{});
    case 5: return f(std::integral_constant<int, 5>{});
    case 6: return f(std::integral_constant<int, 6>{});
    case 7: return f(std::integral_constant<int, 7>{});
    case 8: return f(std::integral_constant<int, 8>{});
    case 9: return f(std::integral_constant<int, 9>{});
    default: return cudaErrorInvalidValue;
  }
}

// Per-device set-up, once, with the device current.  Returns the device
// address of the scratch array (the host-side name g_noalloc_scratch is only a
// stand-in and must never be passed to a kernel).
int setup_device(int dev, double **out) {
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (dev < 0 || dev >= MAX_DEVICES) return nfail(DSEM_ERR_INVALID_ARG, "device index out of range");
  if (g_scratch_ptr[dev]) {
    *out = g_scratch_ptr[dev];
    return DSEM_OK;
  }
  double *ptr = nullptr;
  cudaError_t e = cudaGetSymbolAddress((void **)&ptr, g_noalloc_scratch);
  if (e != cudaSuccess || !ptr)
    return nfail(DSEM_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
  static std::vector<double> table;
  if (table.empty()) {
    table.assign(OPS_TOTAL, 0.0);
    for (int G = GMIN; G <= GMAX; ++G) hostmath::operators(G, &table[ops_off(G)], &table[ops_off(G) + G * (G + 1)]);
  }
  for (int G = GMIN; G <= GMAX; ++G) {
    e = with_G(G, [&](auto g) { return Launch<decltype(g)::value>::set_ops(table.data(), OPS_TOTAL); });
    if (e != cudaSuccess) return nfail(DSEM_ERR_CUDA, std::string("operator tables: ") + cudaGetErrorString(e));
    VolArgs a{};
    e = with_G(G, [&](auto g) { return Launch<decltype(g)::value>::vol(a, 0, true, VOL_PLAIN, nullptr); });
    if (e != cudaSuccess) return nfail(DSEM_ERR_CUDA, std::string("kernel attributes: ") + cudaGetErrorString(e));
  }
  g_scratch_ptr[dev] = ptr;
  *out = ptr;
  return DSEM_OK;
}

// Mortar kernels reading the caller's DSEM_MORTAR_INTS rows directly
// (1-based element ids; elements of one order, slots [elem][face][var][G^2]).
// The rows live in device memory, so they are checked here:
//  - a row with an element outside 1..nel, a face outside 1..6 or an
//    orientation outside 0..7 is skipped and sets bit 2 of the flag;
//  - a row that is not a conforming mortar of this order (len(1..2,1..2) or
//    lenmortar(1..2) other than G, or any conforming(i,j) == 0: a
//    p-nonconforming mortar, which dsem_rhs sends through the L2 projections)
//    is skipped and sets bit 3 of the flag.
__device__ __forceinline__ bool row_ok(const int *r, int nel, int G, int *flag, int pt) {
  const bool ok = r[0] >= 1 && r[0] <= nel && r[1] >= 1 && r[1] <= nel && r[2] >= 1 && r[2] <= 6 && r[3] >= 1 &&
                  r[3] <= 6 && r[10] >= 0 && r[10] <= 7;
  if (!ok) {
    if (pt == 0) atomicOr(flag, 4);
    return false;
  }
  const bool conf = r[4] == G && r[5] == G && r[6] == G && r[7] == G && r[8] == G && r[9] == G && r[13] != 0 &&
                    r[14] != 0 && r[15] != 0 && r[16] != 0;
  if (!conf && pt == 0) atomicOr(flag, 8);
  return conf;
}

template <int G>
__global__ void __launch_bounds__(128) k_face_inv_rows(const int *__restrict__ rows, int nm, int nel, int *flag,
                                                        double *__restrict__ QF, double *__restrict__ FF,
                                                        const double *__restrict__ nh, const double *__restrict__ nrm,
                                                        double gamma) {
  constexpr int G2 = G * G;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)nm * G2) return;
  const int m = (int)(t / G2), pt = (int)(t - (long long)m * G2);
  const int *r = rows + (long long)DSEM_MORTAR_INTS * m;
  if (!row_ok(r, nel, G, flag, pt)) return;
  const long long ms = (long long)(r[0] - 1) * 30 * G2 + (long long)(r[2] - 1) * 5 * G2;
  const long long ss = (long long)(r[1] - 1) * 30 * G2 + (long long)(r[3] - 1) * 5 * G2;
  int si, sj;
  slave_index<G>(r[10], pt % G, pt / G, si, sj);
  const int sp = si + G * sj;
  double Q1[NV], Q2[NV], f[NV];
  for (int v = 0; v < NV; ++v) {
    Q1[v] = QF[ms + v * G2 + pt];
    Q2[v] = QF[ss + v * G2 + sp];
  }
  const long long gp = (long long)m * G2 + pt;
  const double n3[3] = {nh[gp * 3], nh[gp * 3 + 1], nh[gp * 3 + 2]};
  const bool low = (r[2] == 1 || r[2] == 3 || r[2] == 6);
  riemann(n3, nrm[gp], low ? Q2 : Q1, low ? Q1 : Q2, gamma, f);
  const double sgn = r[11] < 0 ? -1.0 : 1.0;
  for (int v = 0; v < NV; ++v) {
    const double avg = (Q1[v] + Q2[v]) * 0.5;
    FF[ms + v * G2 + pt] = f[v];
    FF[ss + v * G2 + sp] = sgn * f[v];
    QF[ms + v * G2 + pt] = avg;
    QF[ss + v * G2 + sp] = avg;
  }
}

template <int G>
__global__ void __launch_bounds__(128) k_face_vis_rows(const int *__restrict__ rows, int nm, int nel, int *flag,
                                                        double *__restrict__ VF, const double *__restrict__ nrm) {
  constexpr int G2 = G * G;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)nm * G2) return;
  const int m = (int)(t / G2), pt = (int)(t - (long long)m * G2);
  const int *r = rows + (long long)DSEM_MORTAR_INTS * m;
  if (!row_ok(r, nel, G, flag, pt)) return;
  const long long ms = (long long)(r[0] - 1) * 30 * G2 + (long long)(r[2] - 1) * 5 * G2;
  const long long ss = (long long)(r[1] - 1) * 30 * G2 + (long long)(r[3] - 1) * 5 * G2;
  int si, sj;
  slave_index<G>(r[10], pt % G, pt / G, si, sj);
  const int sp = si + G * sj;
  const double nm_m = nrm[(long long)m * G2 + pt], nm_s = nrm[(long long)m * G2 + sp];
  for (int v = 0; v < NV; ++v) {
    const double fv1 = VF[ms + v * G2 + pt] / nm_m;
    const double fv2 = VF[ss + v * G2 + sp] / nm_s;
    const double Qs = r[12] < 0 ? -fv2 : fv2;
    const double qb = 0.5 * (fv1 + Qs) * nm_m;
    VF[ms + v * G2 + pt] = qb;
    VF[ss + v * G2 + sp] = r[11] < 0 ? -qb : qb;
  }
}

template <int G>
int run(double *scratch, int nel, int nmort, const int *rows, const double *nh, const double *nrm, const double *JQ,
        const double *jac, const double *gg, const double *gm, double gamma, double re, double pr, double mach,
        double *Qt, cudaStream_t st) {
  constexpr int G2 = G * G, NG = G * G * G;
  const long long nf = (long long)nel * 30 * G2;
  double *QF = scratch, *FF = QF + nf, *VF = FF + nf, *QTI = VF + nf;
  int *flag = reinterpret_cast<int *>(QTI + (long long)nel * 5 * NG);
  cudaError_t e;
#define NK(x)                                                                                       \
  do {                                                                                              \
    e = (x);                                                                                        \
    if (e != cudaSuccess) return nfail(DSEM_ERR_CUDA, std::string(#x ": ") + cudaGetErrorString(e)); \
  } while (0)
  // face slots without a mortar stay zero; the flag starts clear
  NK(cudaMemsetAsync(FF, 0, 2 * nf * sizeof(double), st));
  NK(cudaMemsetAsync(flag, 0, sizeof(int), st));
  TraceArgs ta{JQ, 5LL * NG, jac, QF};
  NK(Launch<G>::trace(ta, nel, st));
  const unsigned nb = (unsigned)(((long long)nmort * G2 + 127) / 128);
  if (nmort > 0) {
    k_face_inv_rows<G><<<nb, 128, 0, st>>>(rows, nmort, nel, flag, QF, FF, nh, nrm, gamma);
    NK(cudaGetLastError());
  }
  VolArgs va{};
  va.JQ = JQ;
  va.sq = 5LL * NG;
  va.jac = jac;
  va.gg = gg;
  va.gm = gm;
  va.QF = QF;
  va.VF = VF;
  va.QTI = QTI;
  va.P.gamma = gamma;
  va.P.re = re;
  va.P.pr = pr;
  va.P.mach = mach;
  phys_recips(va.P);
  NK(Launch<G>::vol(va, nel, true, VOL_PLAIN, st));
  if (nmort > 0) {
    k_face_vis_rows<G><<<nb, 128, 0, st>>>(rows, nmort, nel, flag, VF, nrm);
    NK(cudaGetLastError());
  }
  UpdArgs ua{};
  ua.JQ = const_cast<double *>(JQ);  // not written: update == 0
  ua.gQ = const_cast<double *>(JQ);
  ua.sq = 5LL * NG;
  ua.jac = jac;
  ua.QTI = QTI;
  ua.FF = FF;
  ua.VF = VF;
  ua.QF = QF;
  ua.Qt_out = Qt;
  ua.flag = flag;
  ua.re = re;
  ua.r_re = 1.0 / re;
  ua.update = 0;
  NK(Launch<G>::update(ua, nel, st));
  int h = 0;
  NK(cudaMemcpyAsync(&h, flag, sizeof(int), cudaMemcpyDeviceToHost, st));
  NK(cudaStreamSynchronize(st));
#undef NK
  if (h & 4) return nfail(DSEM_ERR_INVALID_ARG, "dsem_rhs_noalloc: mortar row with an element, face or orientation out of range");
  if (h & 8)
    return nfail(DSEM_ERR_UNSUPPORTED,
                 "dsem_rhs_noalloc: mortar row is not a conforming mortar of order p (lengths or conforming flags)");
  if (h & 1) return nfail(DSEM_ERR_NONFINITE, "NaN or Inf in the right-hand side");
  return DSEM_OK;
}

}  // namespace

extern "C" {

int dsem_rhs_noalloc(int nel, int p, int nmort, const int *mortar, const double *n_hat, const double *norm,
                     const double *JQ, const double *jac, const double *gmetg_diag, const double *gmet_diag,
                     double gamma, double re, double pr, double mach, double *Qt, void *stream) {
  const int G = p + 1;
  if (G < GMIN || G > GMAX) return nfail(DSEM_ERR_INVALID_ARG, "dsem_rhs_noalloc: order p outside 1..8");
  if (nel <= 0 || nmort < 0) return nfail(DSEM_ERR_INVALID_ARG, "dsem_rhs_noalloc: bad element or mortar count");
  if (!JQ || !jac || !gmetg_diag || !gmet_diag || !Qt || (nmort > 0 && (!mortar || !n_hat || !norm)))
    return nfail(DSEM_ERR_INVALID_ARG, "dsem_rhs_noalloc: null device pointer");
  const long long need = (long long)nel * (90LL * G * G + 5LL * G * G * G) + 1;
  if (need > (long long)DSEM_NOALLOC_SCRATCH_DOUBLES)
    return nfail(DSEM_ERR_INVALID_ARG,
                 "dsem_rhs_noalloc: mesh too large for the static scratch (" + std::to_string(need) +
                     " doubles needed, " + std::to_string((long long)DSEM_NOALLOC_SCRATCH_DOUBLES) +
                     " available: nel*(90*(p+1)^2 + 5*(p+1)^3) + 1 must not exceed DSEM_NOALLOC_SCRATCH_DOUBLES)");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return nfail(DSEM_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  double *scratch = nullptr;
  int r = setup_device(dev, &scratch);
  if (r) return r;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // every call memsets, reads the flag back and waits for the stream: none of
  // that may be recorded into a caller's graph
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  e = cudaStreamIsCapturing(st, &cap);
  if (e != cudaSuccess) return nfail(DSEM_ERR_CUDA, std::string("cudaStreamIsCapturing: ") + cudaGetErrorString(e));
  if (cap != cudaStreamCaptureStatusNone)
    return nfail(DSEM_ERR_INVALID_ARG, "dsem_rhs_noalloc: the stream is being captured; call it outside any capture");
  e = with_G(G, [&](auto g) {
    r = run<decltype(g)::value>(scratch, nel, nmort, mortar, n_hat, norm, JQ, jac, gmetg_diag, gmet_diag, gamma, re,
                                pr, mach, Qt, st);
    return cudaSuccess;
  });
  return r;
}

}  // extern "C"
