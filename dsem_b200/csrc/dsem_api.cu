// dsem_api.cu -- C-ABI of include/dsem_gpu.h: context set-up, layout
// conversion, mortar tables, stage orchestration (one CUDA graph per time
// step), diagnostics.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstddef>
#include <cstring>
#include <algorithm>
#include <map>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/dsem_gpu.h"
#include "dsem_ctx.h"
#include "dsem_lobatto.cuh"
#include "dsem_host_math.h"
#include "dsem_launch.h"
#include "dsem_stage.cuh"

using namespace dsem;

namespace {

thread_local std::string g_create_err;

// ---------------------------------------------------------- layout kernels
__global__ void k_pack(const double *__restrict__ src, int ldx, const int *__restrict__ ext, int ext0, int G, int nf,
                       double *__restrict__ dst, int to_internal) {
  // one block per group element; nf fields of G^3 points
  const int k = blockIdx.x;
  const long long L3 = (long long)ldx * ldx * ldx;
  const int NG = G * G * G;
  const long long e = ext[k] - ext0;
  for (int i = threadIdx.x; i < nf * NG; i += blockDim.x) {
    const int v = i / NG, p = i - v * NG;
    const int n = p % G, m = (p / G) % G, l = p / (G * G);
    const long long s = (e * nf + v) * L3 + n + (long long)ldx * (m + (long long)ldx * l);
    const long long d = (long long)k * nf * NG + i;
    if (to_internal)
      dst[d] = src[s];
    else
      dst[s] = src[d];
  }
}

// Per-element partial sums for the diagnostics, one block per element: the
// point terms in parallel, then each sum accumulated by one thread in the
// oracle's loop order: [0..2] sum u^2 w, v^2 w, w^2 w; [3] sum |w|^2 J; [4] sum J.
__global__ void k_diag(const double *__restrict__ JQ, const double *__restrict__ jac, const double *__restrict__ EVB,
                       const double *__restrict__ kew, int G, int nel, int have_grad, double *__restrict__ part) {
  extern __shared__ double sm[];
  const int k = blockIdx.x;
  const int NG = G * G * G;
  double *T = sm;  // [5][NG]
  const double *Q = JQ + (long long)k * 5 * NG;
  const double *J = jac + (long long)k * NG;
  const double *E = EVB + (long long)k * 15 * NG;
  for (int p = threadIdx.x; p < NG; p += blockDim.x) {
    const double q1 = Q[p];
    const double u = Q[NG + p] / q1, v = Q[2 * NG + p] / q1, w = Q[3 * NG + p] / q1;
    const double b = kew[p];
    T[p] = (u * u) * b;
    T[NG + p] = (v * v) * b;
    T[2 * NG + p] = (w * w) * b;
    if (have_grad) {  // energydissipation.f90:19-78
      const double Q1 = Q[p], Q2 = Q[NG + p], Q3 = Q[2 * NG + p], Q4 = Q[3 * NG + p];
      const double jc = J[p];
      const double Qx0 = E[0 * NG + p], Qy0 = E[1 * NG + p], Qz0 = E[2 * NG + p];
      const double Qy1 = E[4 * NG + p], Qz1 = E[5 * NG + p];
      const double Qx2 = E[6 * NG + p], Qz2 = E[8 * NG + p];
      const double Qx3 = E[9 * NG + p], Qy3 = E[10 * NG + p];
      const double udery = ((Qy1 - (Q2 / Q1) * Qy0)) / Q1;
      const double uderz = ((Qz1 - (Q2 / Q1) * Qz0)) / Q1;
      const double vderx = ((Qx2 - (Q3 / Q1) * Qx0)) / Q1;
      const double vderz = ((Qz2 - (Q3 / Q1) * Qz0)) / Q1;
      const double wderx = ((Qx3 - (Q4 / Q1) * Qx0)) / Q1;
      const double wdery = ((Qy3 - (Q4 / Q1) * Qy0)) / Q1;
      const double c1 = (wdery - vderz) / jc, c2 = (uderz - wderx) / jc, c3 = (vderx - udery) / jc;
      double vort = c1 * c1 + c2 * c2 + c3 * c3;
      vort = vort / jc;
      T[3 * NG + p] = vort;
      T[4 * NG + p] = 1.0 / jc;
    }
  }
  __syncthreads();
  const int f = threadIdx.x;
  if (f < 3 || (f < 5 && have_grad)) {
    const double *t = T + f * NG;
    double acc = 0.0;
    if (f < 3) {
      for (int i = 0; i < G; ++i)
        for (int j = 0; j < G; ++j)
          for (int l = 0; l < G; ++l) acc = acc + t[i + G * (j + G * l)];
    } else {
      for (int l = 0; l < G; ++l)
        for (int m = 0; m < G; ++m)
          for (int n = 0; n < G; ++n) acc = acc + t[l + G * (m + G * n)];
    }
    part[(long long)k * 5 + f] = acc;
  } else if (f < 5) {
    part[(long long)k * 5 + f] = 0.0;
  }
}

}  // namespace


namespace {

int fail(dsem_ctx *c, int code, const std::string &msg) {
  if (c)
    c->err = msg;
  else
    g_create_err = msg;
  return code;
}
int cuda_fail(dsem_ctx *c, cudaError_t e, const char *where) {
  return fail(c, DSEM_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}
#define CK(call)                                          \
  do {                                                    \
    cudaError_t e_ = (call);                              \
    if (e_ != cudaSuccess) return cuda_fail(c, e_, #call); \
  } while (0)

void rkcoefs(dsem_ctx *c, int iord) {  // Independentroutines/baselib.f90:86-160
  for (int i = 0; i < 5; ++i) c->ark[i] = c->brk[i] = c->crk[i] = 0.0;
  if (iord == 3) {
    c->kord = 3;
    c->ark[1] = -5.0 / 9.0;
    c->ark[2] = -153.0 / 128.0;
    c->brk[1] = 1.0 / 3.0;
    c->brk[2] = 3.0 / 4.0;
    c->crk[0] = 1.0 / 3.0;
    c->crk[1] = 15.0 / 16.0;
    c->crk[2] = 8.0 / 15.0;
  } else if (iord == 2) {
    c->kord = 2;
    c->ark[1] = -1.0;
    c->brk[1] = 1.0;
    c->crk[0] = 1.0;
    c->crk[1] = 0.5;
  } else if (iord == 1) {
    c->kord = 1;
    c->crk[0] = 1.0;
  } else {
    c->kord = 5;
    c->ark[1] = -0.4178904745;
    c->ark[2] = -1.192151694643;
    c->ark[3] = -1.697784692471;
    c->ark[4] = -1.514183444257;
    c->brk[1] = 0.1496590219993;
    c->brk[2] = 0.3704009573644;
    c->brk[3] = 0.6222557631345;
    c->brk[4] = 0.9582821306748;
    c->crk[0] = 0.1496590219993;
    c->crk[1] = 0.3792103129999;
    c->crk[2] = 0.8229550293869;
    c->crk[3] = 0.6994504559488;
    c->crk[4] = 0.1530572479681;
  }
}

int upload_ops(dsem_ctx *c) {
  static std::vector<double> table;
  if (table.empty()) {
    table.assign(OPS_TOTAL, 0.0);
    for (int G = GMIN; G <= GMAX; ++G) {
      const int L = G + 1;
      hostmath::operators(G, &table[ops_off(G)], &table[ops_off(G) + G * L]);
    }
  }
  for (int G = GMIN; G <= GMAX; ++G) {
    cudaError_t e = with_G(G, [&](auto g) { return Launch<decltype(g)::value>::set_ops(table.data(), OPS_TOTAL); });
    if (e != cudaSuccess) return cuda_fail(c, e, "set_ops");
  }
  return DSEM_OK;
}

// Runs f(j, stream) for jobs j = 0..n-1. With more than one job each gets its
// own stream, forked from the context stream and joined back into it, so that
// independent order groups (and mortar lists) overlap on the device and form
// parallel branches of a captured graph.
template <class F> int fork_jobs(dsem_ctx *c, size_t n, F &&f) {
  if (n <= 1) {
    for (size_t j = 0; j < n; ++j) {
      const int r = f(j, c->st);
      if (r) return r;
    }
    return DSEM_OK;
  }
  if (n > c->aux.size()) return fail(c, DSEM_ERR_INVALID_ARG, "more parallel jobs than auxiliary streams");
  CK(cudaEventRecord(c->ev_fork, c->st));
  for (size_t j = 0; j < n; ++j) {
    CK(cudaStreamWaitEvent(c->aux[j], c->ev_fork, 0));
    const int r = f(j, c->aux[j]);
    if (r) return r;
    CK(cudaEventRecord(c->ev_join[j], c->aux[j]));
  }
  for (size_t j = 0; j < n; ++j) CK(cudaStreamWaitEvent(c->st, c->ev_join[j], 0));
  return DSEM_OK;
}

int vol_mode(const dsem_ctx *c, bool save) {
  if (c->shock) return save ? VOL_EV_SAVE : VOL_EV;
  return save ? VOL_SAVE : VOL_PLAIN;
}

// The four parts of one evaluation of Fluxes + the flux divergence (+ the
// update when kk > 0).  The update reads dt per case from d_dtc (written before
// the stage is enqueued or the graph replayed).
// physical constants of the boundary kernels
static dsem::BndPhys bnd_phys(const dsem_ctx *c) {
  dsem::BndPhys P;
  P.gamma = c->P.gamma;
  P.twall = c->twall;
  P.cv = c->P.mach * c->P.mach * c->P.gamma * (c->P.gamma - 1.0);
  P.r_cv = 1.0 / P.cv;
  return P;
}

int enqueue_face_inv(dsem_ctx *c, long long *launches) {
  if ((c->bnd_need_twall && !c->bnd_twall_set) || (c->bnd_need_ext && !c->bnd_ext_set))
    return fail(c, DSEM_ERR_INVALID_ARG,
                "boundary faces need dsem_set_boundary first (twall for isothermal walls, external states for "
                "inflow/outflow)");
  const double gamma = c->P.gamma;
  const size_t nml = c->mlists.size(), nnj = nml + (c->nnc > 0 ? 1 : 0), nfj = nnj + c->blists.size();
  const dsem::BndPhys BP = bnd_phys(c);
  int r = fork_jobs(c, nfj, [&](size_t j, cudaStream_t st) -> int {
    if (j < nml) {
      auto &ml = c->mlists[j];
      CK(with_G(ml.G, [&](auto g) {
        return Launch<decltype(g)::value>::face_inv(ml.mc, ml.n, c->QF, c->FF, ml.nh, ml.nrm, gamma, st);
      }));
    } else if (j >= nnj) {  // boundary faces: their master face slots only
      auto &bl = c->blists[j - nnj];
      CK(with_G(bl.G, [&](auto g) {
        return Launch<decltype(g)::value>::face_bnd_inv(bl.mb, bl.n, c->QF, c->FF, bl.nh, bl.nrm, bl.qext, BP, st);
      }));
    } else {
      k_face_nc_inv<<<c->nnc, 128, 0, st>>>(c->nc, c->QF, c->FF, c->nc_nh, c->nc_nrm, c->nc_mats, gamma);
      CK(cudaGetLastError());
    }
    return DSEM_OK;
  });
  if (r) return r;
  *launches += (long long)nfj;
  if (c->ncut > 0) {
    CK(with_G(c->cut_G, [&](auto g) {
      return Launch<decltype(g)::value>::face_inv_cut(c->cut, c->ncut, c->QF, c->FF, c->ghost, c->cut_nh, c->cut_nrm,
                                                      gamma, c->st);
    }));
    ++*launches;
  }
  return DSEM_OK;
}

// volume kernel arguments of one order group
VolArgs vol_args(const dsem_ctx *c, const Group &g) {
  VolArgs a{};
  a.JQ = c->JQ + g.q0;
  a.sq = 5LL * g.G * g.G * g.G;
  a.jac = g.jac;
  a.gg = g.gg;
  a.gm = g.gm;
  a.muhg = g.muhg;
  a.QF = c->QF + g.f0;
  a.VF = c->VF + g.f0;
  a.QTI = c->QTI + g.q0;
  a.EVB = g.EVB;
  a.P = c->P;
  a.ecase = g.ecase;
  a.rec = c->d_rec;
  a.nuhg = c->les ? g.nuhg : nullptr;
  return a;
}

int enqueue_vol(dsem_ctx *c, bool save, long long *launches) {
  const int mode = vol_mode(c, save);
  int r = fork_jobs(c, c->groups.size(), [&](size_t j, cudaStream_t st) -> int {
    auto &g = c->groups[j];
    const VolArgs a = vol_args(c, g);
    CK(with_G(g.G, [&](auto gg) {
      return Launch<decltype(gg)::value>::vol(a, g.nel, g.diag, mode, st, c->vol_variant[g.G]);
    }));
    return DSEM_OK;
  });
  if (r) return r;
  *launches += (long long)c->groups.size();
  return DSEM_OK;
}

int enqueue_face_vis(dsem_ctx *c, long long *launches) {
  const size_t nml = c->mlists.size(), nnj = nml + (c->nnc > 0 ? 1 : 0), nfj = nnj + c->blists.size();
  int r = fork_jobs(c, nfj, [&](size_t j, cudaStream_t st) -> int {
    if (j < nml) {
      auto &ml = c->mlists[j];
      CK(with_G(ml.G, [&](auto g) { return Launch<decltype(g)::value>::face_vis(ml.mc, ml.n, c->VF, ml.nrm, st); }));
    } else if (j >= nnj) {
      auto &bl = c->blists[j - nnj];
      CK(with_G(bl.G, [&](auto g) {
        return Launch<decltype(g)::value>::face_bnd_vis(bl.mb, bl.n, c->VF, bl.nrm, bl.fvext, st);
      }));
    } else {
      k_face_nc_vis<<<c->nnc, 128, 0, st>>>(c->nc, c->VF, c->nc_nrm, c->nc_mats);
      CK(cudaGetLastError());
    }
    return DSEM_OK;
  });
  if (r) return r;
  *launches += (long long)nfj;
  if (c->ncut > 0) {
    CK(with_G(c->cut_G, [&](auto g) {
      return Launch<decltype(g)::value>::face_vis_cut(c->cut, c->ncut, c->VF, c->ghost, c->cut_nrm, c->st);
    }));
    ++*launches;
  }
  return DSEM_OK;
}

// update kernel arguments of one order group for stage kk (0: Qt only)
UpdArgs upd_args(const dsem_ctx *c, const Group &g, int kk, double *qt_out) {
  UpdArgs u{};
  u.JQ = c->JQ + g.q0;
  u.gQ = c->gQ + g.q0;
  u.sq = 5LL * g.G * g.G * g.G;
  u.jac = g.jac;
  u.QTI = c->QTI + g.q0;
  u.FF = c->FF + g.f0;
  u.VF = c->VF + g.f0;
  u.QF = c->QF + g.f0;
  u.Qt_out = qt_out ? qt_out + g.q0 : nullptr;
  u.flag = c->flag;
  u.re = c->P.re;
  u.r_re = c->P.r_re;
  u.update = kk > 0;
  u.first = kk == 1;
  u.ark = kk > 0 ? c->ark[kk - 1] : 0.0;
  u.crk = kk > 0 ? c->crk[kk - 1] : 0.0;
  u.ecase = g.ecase;
  u.rec = c->d_rec;
  u.dtc = c->d_dtc;
  return u;
}

// the update kernel of group g averages the raw viscous face fluxes itself (k_update<G, true>;
// c->fuse_vis contexts, no k_face_vis before it)
void fuse_vis_args(const dsem_ctx *c, const Group &g, UpdArgs &u) {
  for (const auto &ml : c->mlists)
    if (ml.G == g.G) {
      u.fmc = g.fmc;
      u.VFr = c->VF;
      u.vnrm = ml.nrm;
    }
}

// fuse_vis: the update kernel averages the raw viscous face fluxes itself (c->fuse_vis
// contexts; no enqueue_face_vis before it)
int enqueue_update(dsem_ctx *c, int kk, double *qt_out, long long *launches, bool fuse_vis = false) {
  int r = fork_jobs(c, c->groups.size(), [&](size_t j, cudaStream_t st) -> int {
    auto &g = c->groups[j];
    UpdArgs u = upd_args(c, g, kk, qt_out);
    if (fuse_vis) fuse_vis_args(c, g, u);
    CK(with_G(g.G, [&](auto gg) { return Launch<decltype(gg)::value>::update(u, g.nel, st); }));
    return DSEM_OK;
  });
  if (r) return r;
  *launches += (long long)c->groups.size();
  return DSEM_OK;
}

// the Lobatto arrays of the stage about to run (its state and averaged face
// traces) into c->QLB (d%Qlgg/Qglg/Qggl of the last stage, for the restart file)
int enqueue_lob_keep(dsem_ctx *c, long long *launches) {
  const int r = fork_jobs(c, c->groups.size(), [&](size_t j, cudaStream_t st) -> int {
    auto &g = c->groups[j];
    LobArgs a{};
    a.JQ = c->JQ + g.q0;
    a.sq = 5LL * g.G * g.G * g.G;
    a.jac = g.jac;
    a.QF = c->QF + g.f0;
    a.QLB = c->QLB + g.l0;
    CK(with_G(g.G, [&](auto gg) { return Launch<decltype(gg)::value>::lob_keep(a, g.nel, st); }));
    return DSEM_OK;
  });
  if (r) return r;
  *launches += (long long)c->groups.size();
  return DSEM_OK;
}

// fuse_vis (dsem_step): on c->fuse_vis contexts the update kernel averages the viscous
// face fluxes and k_face_vis is not launched (VF keeps the raw fluxes after the stage)
int enqueue_stage(dsem_ctx *c, int kk, bool save, double *qt_out, long long *launches, bool fuse_vis = false) {
  int r;
  fuse_vis = fuse_vis && c->fuse_vis;
  if ((r = enqueue_face_inv(c, launches))) return r;
  if (kk == c->kord && c->keep_lob && (r = enqueue_lob_keep(c, launches))) return r;
  if ((r = enqueue_vol(c, save, launches))) return r;
  if (!fuse_vis && (r = enqueue_face_vis(c, launches))) return r;
  return enqueue_update(c, kk, qt_out, launches, fuse_vis);
}

int enqueue_ev(dsem_ctx *c, long long *launches, const double *jq = nullptr) {
  if (!jq) jq = c->JQ;
  const int r = fork_jobs(c, c->groups.size(), [&](size_t j, cudaStream_t st) -> int {
    auto &g = c->groups[j];
    EvArgs a{};
    a.JQ = jq + g.q0;
    a.sq = 5LL * g.G * g.G * g.G;
    a.jac = g.jac;
    a.hd = g.hd;
    a.EVB = g.EVB;
    a.muhg = g.muhg;
    a.sens = c->les_sensors ? g.sens : nullptr;
    a.valid = c->ev_grad_valid ? 1 : 0;
    a.P = c->P;
    a.ecase = g.ecase;
    a.rec = c->d_rec;
    CK(with_G(g.G, [&](auto gg) { return Launch<decltype(gg)::value>::ev(a, g.nel, st); }));
    return DSEM_OK;
  });
  if (r) return r;
  *launches += (long long)c->groups.size();
  return DSEM_OK;
}

// Smagorinsky viscosity from the last Fluxes call's gradients (tstep.f90:40-43)
int enqueue_les(dsem_ctx *c, long long *launches, const double *jq = nullptr) {
  if (!jq) jq = c->JQ;
  const int r = fork_jobs(c, c->groups.size(), [&](size_t j, cudaStream_t st) -> int {
    auto &g = c->groups[j];
    LesArgs a{};
    a.JQ = jq + g.q0;
    a.sq = 5LL * g.G * g.G * g.G;
    a.jac = g.jac;
    a.hd = g.hd;
    a.EVB = g.EVB;
    a.nuhg = g.nuhg;
    a.sens = g.sens;
    a.sensors = c->les_sensors;
    a.valid = c->grad_valid ? 1 : 0;
    a.re = c->P.re;
    a.cs = c->les_cs;
    a.numax = c->les_numax;
    a.ecase = g.ecase;
    a.rec = c->d_rec;
    CK(with_G(g.G, [&](auto gg) { return Launch<decltype(gg)::value>::les(a, g.nel, st); }));
    return DSEM_OK;
  });
  if (r) return r;
  *launches += (long long)c->groups.size();
  return DSEM_OK;
}

int enqueue_traces(dsem_ctx *c, long long *launches) {
  const int r = fork_jobs(c, c->groups.size(), [&](size_t j, cudaStream_t st) -> int {
    auto &g = c->groups[j];
    TraceArgs a{};
    a.JQ = c->JQ + g.q0;
    a.sq = 5LL * g.G * g.G * g.G;
    a.jac = g.jac;
    a.QF = c->QF + g.f0;
    CK(with_G(g.G, [&](auto gg) { return Launch<decltype(gg)::value>::trace(a, g.nel, st); }));
    return DSEM_OK;
  });
  if (r) return r;
  *launches += (long long)c->groups.size();
  c->traces_valid = true;
  return DSEM_OK;
}

// one full time step (tstep.f90:36-116): EV, g_Q = 0 (folded into stage 1), kord stages
int enqueue_step(dsem_ctx *c, bool save_last, long long *launches) {
  if (c->shock) {
    int r = enqueue_ev(c, launches);
    if (r) return r;
  }
  if (c->les) {
    int r = enqueue_les(c, launches);
    if (r) return r;
  }
  for (int kk = 1; kk <= c->kord; ++kk) {
    int r = enqueue_stage(c, kk, save_last && kk == c->kord, nullptr, launches, true);
    if (r) return r;
  }
  return DSEM_OK;
}

int ensure_stage_buf(dsem_ctx *c, int ldx, int nf) {
  const size_t need = (size_t)c->ngrid * nf * ldx * ldx * ldx;
  if (need > c->nstage) {
    if (c->stage) cudaFree(c->stage);
    c->stage = nullptr;
    CK(cudaMalloc(&c->stage, need * sizeof(double)));
    c->nstage = need;
  }
  return DSEM_OK;
}

int check_ldx(dsem_ctx *c, int ldx) {
  for (auto &g : c->groups)
    if (ldx < g.G) return fail(c, DSEM_ERR_INVALID_ARG, "ldx smaller than the number of Gauss points");
  return DSEM_OK;
}

// device internal [group elements][nf][G^3] <-> caller [ngrid][nf][ldx^3]
int unpack_to_host(dsem_ctx *c, const double *dev_internal, double *host, int ldx, int nf, const std::vector<long long> &offs) {
  int r = ensure_stage_buf(c, ldx, nf);
  if (r) return r;
  const size_t n = (size_t)c->ngrid * nf * ldx * ldx * ldx;
  CK(cudaMemsetAsync(c->stage, 0, n * sizeof(double), c->st));
  for (size_t gi = 0; gi < c->groups.size(); ++gi) {
    auto &g = c->groups[gi];
    if (g.nel == 0) continue;
    k_pack<<<g.nel, 256, 0, c->st>>>(dev_internal + offs[gi], ldx, g.int2ext, 0, g.G, nf, c->stage, 0);
    CK(cudaGetLastError());
  }
  CK(cudaMemcpyAsync(host, c->stage, n * sizeof(double), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return DSEM_OK;
}

std::vector<long long> state_offs(const dsem_ctx *c) {
  std::vector<long long> o;
  for (auto &g : c->groups) o.push_back(g.q0);
  return o;
}

int check_flag(dsem_ctx *c) {
  int h = 0;
  CK(cudaMemcpyAsync(&h, c->flag, sizeof(int), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  if (h & 1) return fail(c, DSEM_ERR_NONFINITE, "NaN or Inf in the stage right-hand side");
  return DSEM_OK;
}

}  // namespace

// =================================================================== C-ABI
namespace {

// The cases of a context, each a caller descriptor with its own padding ldx;
// caller element e of case k is context element case_el0[k] + e (no copy of
// the caller's arrays is made).
struct MeshSet {
  std::vector<const dsem_mesh_desc *> m;
  std::vector<int> el0, mo0;  // first element / mortar of each case (+ totals)
  double snap = 0.0;          // off-diagonal metric entries up to snap x the point's largest diagonal count as 0
  int case_of(int e) const {
    return (int)(std::upper_bound(el0.begin(), el0.end(), e) - el0.begin()) - 1;
  }
  int ngrid() const { return el0.back(); }
  int nmort() const { return mo0.back(); }
  int G(int e) const {
    const int k = case_of(e);
    return m[k]->ncg[3 * (e - el0[k])];
  }
  // caller point (n, mm, l) of element e: descriptor, flat point index, ldx
  const dsem_mesh_desc *at(int e, int n, int mm, int l, size_t &q) const {
    const int k = case_of(e);
    const size_t ld = (size_t)m[k]->ldx;
    q = (size_t)(e - el0[k]) * ld * ld * ld + n + ld * (mm + ld * l);
    return m[k];
  }
};

int setup_ctx(dsem_ctx *c, const MeshSet &ms);

int check_desc(const dsem_mesh_desc *m) {
  if (m->ngrid <= 0 || m->nmort < 0 || m->ldx <= 0 || !m->ncg || !m->jacob || !m->gmetg || !m->gmet ||
      (m->nmort > 0 && (!m->mortar || !m->n_hat || !m->norm)))
    return fail(nullptr, DSEM_ERR_INVALID_ARG, "incomplete mesh descriptor");
  for (int e = 0; e < m->ngrid; ++e) {
    const int G = m->ncg[3 * e];
    if (m->ncg[3 * e + 1] != G || m->ncg[3 * e + 2] != G)
      return fail(nullptr, DSEM_ERR_UNSUPPORTED, "anisotropic element orders are not supported");
    if (G < GMIN || G > GMAX) return fail(nullptr, DSEM_ERR_UNSUPPORTED, "element order outside 1..8");
    if (m->ldx < G + 1) return fail(nullptr, DSEM_ERR_INVALID_ARG, "ldx must be at least ncg+1");
  }
  return DSEM_OK;
}

int create_ctx(const MeshSet &ms, const dsem_phys *ph, const std::vector<double> &re, dsem_ctx **out) {
  dsem_ctx *c = new dsem_ctx();
  cudaGetDevice(&c->dev);
  if (cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking) != cudaSuccess) {
    delete c;
    return fail(nullptr, DSEM_ERR_CUDA, "cudaStreamCreate failed (no usable CUDA device?)");
  }
  c->ngrid = ms.ngrid();
  c->nmort = ms.nmort();
  c->P.gamma = ph->gamma;
  c->P.re = re[0];
  c->P.pr = ph->pr;
  c->P.mach = ph->mach;
  c->P.cmu = ph->cmu;
  c->P.mumax = ph->mumax;
  c->P.ducros = (ph->shock & 2) ? 1 : 0;
  phys_recips(c->P);
  c->shock = ph->shock ? 1 : 0;
  c->iord = ph->iord;
  rkcoefs(c, ph->iord);
  c->ncase = (int)ms.m.size();
  c->case_el0 = ms.el0;
  c->case_re = re;
  c->case_dt.assign(c->ncase, 0.0);
  c->case_prestep.assign(c->ncase, 0.0);
  const int r = setup_ctx(c, ms);
  if (r) {
    g_create_err = c->err;
    dsem_destroy(c);
    return r;
  }
  *out = c;
  return DSEM_OK;
}

}  // namespace

// error text of calls made without a context (read by dsem_last_error(NULL))
void dsem_set_thread_error(const std::string &msg) { g_create_err = msg; }

extern "C" {

const char *dsem_last_error(const dsem_ctx *c) { return c ? c->err.c_str() : g_create_err.c_str(); }

int dsem_create(const dsem_mesh_desc *m, const dsem_phys *ph, dsem_ctx **out) {
  if (!m || !ph || !out) return fail(nullptr, DSEM_ERR_INVALID_ARG, "null argument");
  *out = nullptr;
  int r = check_desc(m);
  if (r) return r;
  MeshSet ms;
  ms.m = {m};
  ms.el0 = {0, m->ngrid};
  ms.mo0 = {0, m->nmort};
  return create_ctx(ms, ph, {ph->re}, out);
}

int dsem_create_snapped(const dsem_mesh_desc *m, const dsem_phys *ph, double metric_snap, dsem_ctx **out) {
  if (!m || !ph || !out) return fail(nullptr, DSEM_ERR_INVALID_ARG, "null argument");
  if (!(metric_snap >= 0.0 && metric_snap < 1e-6))
    return fail(nullptr, DSEM_ERR_INVALID_ARG, "metric_snap must lie in [0, 1e-6)");
  *out = nullptr;
  int r = check_desc(m);
  if (r) return r;
  MeshSet ms;
  ms.m = {m};
  ms.el0 = {0, m->ngrid};
  ms.mo0 = {0, m->nmort};
  ms.snap = metric_snap;
  return create_ctx(ms, ph, {ph->re}, out);
}

int dsem_create_batch(int ncase, const dsem_mesh_desc *meshes, const dsem_phys *phys, dsem_ctx **out) {
  if (!meshes || !phys || !out || ncase <= 0) return fail(nullptr, DSEM_ERR_INVALID_ARG, "null argument or ncase < 1");
  *out = nullptr;
  MeshSet ms;
  ms.el0 = {0};
  ms.mo0 = {0};
  std::vector<double> re;
  for (int k = 0; k < ncase; ++k) {
    const dsem_mesh_desc *m = &meshes[k];
    const dsem_phys *p = &phys[k];
    int r = check_desc(m);
    if (r) return r;
    if (p->gamma != phys[0].gamma || p->pr != phys[0].pr || p->mach != phys[0].mach || p->cmu != phys[0].cmu ||
        p->mumax != phys[0].mumax || p->shock != phys[0].shock || p->iord != phys[0].iord)
      return fail(nullptr, DSEM_ERR_UNSUPPORTED,
                  "cases of one batch must share gamma, pr, mach, cmu, mumax, shock and iord (re and dt may differ)");
    if (!(p->re > 0.0)) return fail(nullptr, DSEM_ERR_INVALID_ARG, "re must be positive");
    if ((long long)ms.el0.back() + m->ngrid > 0x7fffffffLL || (long long)ms.mo0.back() + m->nmort > 0x7fffffffLL)
      return fail(nullptr, DSEM_ERR_INVALID_ARG, "batch too large");
    ms.m.push_back(m);
    ms.el0.push_back(ms.el0.back() + m->ngrid);
    ms.mo0.push_back(ms.mo0.back() + m->nmort);
    re.push_back(p->re);
  }
  return create_ctx(ms, &phys[0], re, out);
}

}  // extern "C"

namespace {
int setup_ctx(dsem_ctx *c, const MeshSet &ms) {
  int r = upload_ops(c);
  if (r) return r;
  const int ngrid = ms.ngrid();

  // ---- groups: elements sorted by order
  c->ext_group.assign(ngrid, -1);
  c->ext_k.assign(ngrid, -1);
  long long q0 = 0, f0 = 0, e0 = 0;
  for (int G = GMIN; G <= GMAX; ++G) {
    std::vector<int> ids;
    for (int e = 0; e < ngrid; ++e)
      if (ms.G(e) == G) ids.push_back(e);
    if (ids.empty()) continue;
    Group g;
    g.G = G;
    g.nel = (int)ids.size();
    g.e0 = e0;
    g.q0 = q0;
    g.f0 = f0;
    const int L = G + 1, NG = G * G * G, NL = L * G * G;
    // metric layout: diagonal when every off-diagonal entry is zero (with ms.snap > 0: at
    // most snap times the largest diagonal entry of its point, dsem_create_snapped)
    bool diag = true;
    auto off_zero = [&](const double *g3, int i, int j) {
      const double x = std::fabs(g3[i + 3 * j]);
      if (ms.snap <= 0.0) return x == 0.0;
      const double scale = std::max(std::fabs(g3[0]), std::max(std::fabs(g3[4]), std::fabs(g3[8])));
      return x <= ms.snap * scale;
    };
    for (int e : ids) {
      for (int l = 0; l < L && diag; ++l)
        for (int mm = 0; mm < L && diag; ++mm)
          for (int n = 0; n < L && diag; ++n) {
            size_t q;
            const dsem_mesh_desc *m = ms.at(e, n, mm, l, q);
            if (n < G && mm < G && l < G)
              for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j)
                  if (i != j && !off_zero(m->gmetg + q * 9, i, j)) diag = false;
            const int idx[3] = {n, mm, l};
            for (int d = 0; d < 3; ++d) {
              bool ok = true;
              for (int a = 0; a < 3; ++a)
                if (idx[a] >= (a == d ? L : G)) ok = false;
              if (!ok) continue;
              for (int j = 0; j < 3; ++j)
                if (j != d && !off_zero(m->gmet + q * 9, d, j)) diag = false;
            }
          }
      if (!diag) break;
    }
    g.diag = diag;
    std::vector<double> jac((size_t)g.nel * NG), hd((size_t)g.nel * NG);
    std::vector<double> gg((size_t)g.nel * (diag ? 3 : 9) * NG), gmv((size_t)g.nel * (diag ? 3 : 9) * NL);
    std::vector<int> ec(ids.size());
    g.case_lo.assign(c->ncase, 0);
    g.case_hi.assign(c->ncase, 0);
    for (int k = 0; k < g.nel; ++k) {
      const int e = ids[k];
      const int cs = ms.case_of(e);
      ec[k] = cs;
      if (g.case_hi[cs] == 0) g.case_lo[cs] = k;  // ids increase and cases are contiguous
      g.case_hi[cs] = k + 1;
      c->ext_group[e] = (int)c->groups.size();
      c->ext_k[e] = k;
      for (int l = 0; l < G; ++l)
        for (int mm = 0; mm < G; ++mm)
          for (int n = 0; n < G; ++n) {
            size_t q;
            const dsem_mesh_desc *m = ms.at(e, n, mm, l, q);
            const int p = n + G * (mm + G * l);
            jac[(size_t)k * NG + p] = m->jacob[q];
            hd[(size_t)k * NG + p] =  // delta_g (turbulence/staticSmago/staticSmag.f90:191-201)
                std::pow(std::fabs(1.0 / m->jacob[q]), 1.0 / 3.0) / std::pow((double)(G * G * G), 1.0 / 3.0);
            for (int i = 0; i < 3; ++i)
              for (int j = 0; j < 3; ++j) {
                const double v = m->gmetg[q * 9 + i + 3 * j];
                if (diag) {
                  if (i == j) gg[((size_t)k * 3 + i) * NG + p] = v;
                } else {
                  gg[((size_t)k * NG + p) * 9 + i + 3 * j] = v;
                }
              }
          }
      for (int d = 0; d < 3; ++d) {
        const int ext[3] = {d == 0 ? L : G, d == 1 ? L : G, d == 2 ? L : G};
        for (int l = 0; l < ext[2]; ++l)
          for (int mm = 0; mm < ext[1]; ++mm)
            for (int n = 0; n < ext[0]; ++n) {
              size_t q;
              const dsem_mesh_desc *m = ms.at(e, n, mm, l, q);
              const int pl = d == 0 ? n + L * (mm + G * l) : (d == 1 ? n + G * (mm + L * l) : n + G * (mm + G * l));
              if (diag) {
                gmv[((size_t)k * 3 + d) * NL + pl] = m->gmet[q * 9 + d + 3 * d];
              } else {
                for (int j = 0; j < 3; ++j) gmv[(((size_t)k * 3 + d) * NL + pl) * 3 + j] = m->gmet[q * 9 + d + 3 * j];
              }
            }
      }
    }
    CK(cudaMalloc(&g.jac, jac.size() * sizeof(double)));
    CK(cudaMalloc(&g.hd, hd.size() * sizeof(double)));
    CK(cudaMalloc(&g.gg, gg.size() * sizeof(double)));
    CK(cudaMalloc(&g.gm, gmv.size() * sizeof(double)));
    CK(cudaMemcpy(g.jac, jac.data(), jac.size() * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(g.hd, hd.data(), hd.size() * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(g.gg, gg.data(), gg.size() * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(g.gm, gmv.data(), gmv.size() * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMalloc(&g.muhg, (size_t)g.nel * NG * sizeof(double)));
    CK(cudaMemset(g.muhg, 0, (size_t)g.nel * NG * sizeof(double)));
    CK(cudaMalloc(&g.EVB, (size_t)g.nel * 15 * NG * sizeof(double)));
    CK(cudaMemset(g.EVB, 0, (size_t)g.nel * 15 * NG * sizeof(double)));
    CK(cudaMalloc(&g.int2ext, ids.size() * sizeof(int)));
    CK(cudaMemcpy(g.int2ext, ids.data(), ids.size() * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMalloc(&g.ecase, ec.size() * sizeof(int)));
    CK(cudaMemcpy(g.ecase, ec.data(), ec.size() * sizeof(int), cudaMemcpyHostToDevice));
    std::vector<double> kw(NG);
    hostmath::ke_weights(G, kw.data());
    CK(cudaMalloc(&g.kew, NG * sizeof(double)));
    CK(cudaMemcpy(g.kew, kw.data(), NG * sizeof(double), cudaMemcpyHostToDevice));
    c->groups.push_back(g);
    q0 += 5LL * g.nel * NG;
    f0 += 30LL * g.nel * G * G;
    e0 += g.nel;
  }
  c->nq = (size_t)q0;
  c->nface = (size_t)f0;

  // ---- mortars
  std::vector<MortarCut> cuts;
  std::vector<int> cut_ghost;
  std::vector<double> cut_nh, cut_nrm;
  int cut_G = 0;
  std::vector<std::vector<MortarC>> mcs(GMAX + 1);
  std::vector<MortarNC> ncs;
  std::vector<double> nc_nh, nc_nrm, mats;
  std::map<long long, std::pair<int, int>> mat_off;
  std::vector<std::vector<double>> nhs(GMAX + 1), nrs(GMAX + 1);
  std::vector<std::vector<dsem::MortarB>> bms(GMAX + 1);
  std::vector<std::vector<double>> bnhs(GMAX + 1), bnrs(GMAX + 1);
  std::vector<std::vector<int>> bids(GMAX + 1);
  for (int cs = 0; cs < c->ncase; ++cs) {
  const dsem_mesh_desc *m = ms.m[cs];
  const int ldx = m->ldx;
  for (int j = 0; j < m->nmort; ++j) {
    const int *t = m->mortar + (size_t)DSEM_MORTAR_INTS * j;
    if (t[0] < 0 || t[1] < 0) {  // cut mortar: the side with id -(g+1) is ghost face g (another shard)
      if (c->ncase != 1) return fail(c, DSEM_ERR_UNSUPPORTED, "cut mortars are not supported in an ensemble");
      if (t[0] < 0 && t[1] < 0) return fail(c, DSEM_ERR_INVALID_ARG, "a cut mortar needs one local side");
      const bool lm = t[0] > 0;
      const int lid = (lm ? t[0] : t[1]) - 1, g = -(lm ? t[1] : t[0]) - 1;
      if (lid < 0 || lid >= m->ngrid) return fail(c, DSEM_ERR_INVALID_ARG, "mortar id out of range");
      const int f1 = t[2], f2 = t[3], orient = t[10];
      if (f1 < 1 || f1 > 6 || f2 < 1 || f2 > 6 || orient < 0 || orient > 7)
        return fail(c, DSEM_ERR_INVALID_ARG, "bad mortar face or orientation");
      const int G = ms.G(lid), G2 = G * G;
      if (!(t[13] && t[14] && t[15] && t[16]) || t[4] != G || t[5] != G || t[6] != G || t[7] != G || t[8] != G ||
          t[9] != G)
        return fail(c, DSEM_ERR_UNSUPPORTED, "cut mortars must be conforming");
      if (cut_G && cut_G != G) return fail(c, DSEM_ERR_UNSUPPORTED, "cut mortars of one order only");
      cut_G = G;
      const int lf = lm ? f1 : f2;
      MortarCut mc;
      mc.ls = c->groups[c->ext_group[lid]].f0 + (long long)c->ext_k[lid] * 30 * G2 + (long long)(lf - 1) * 5 * G2;
      mc.go = (long long)g * 5 * G2;
      mc.geo = (int)cuts.size();
      const bool low = (f1 == 1 || f1 == 3 || f1 == 6);
      mc.flags = orient | ((t[11] < 0) << 3) | ((t[12] < 0) << 4) | (low << 5) | ((lm ? 1 : 0) << 6);
      cuts.push_back(mc);
      cut_ghost.push_back(g);
      for (int jj = 0; jj < G; ++jj)
        for (int i = 0; i < G; ++i) {
          const size_t q = (size_t)j * ldx * ldx + i + (size_t)ldx * jj;
          cut_nrm.push_back(m->norm[q]);
          for (int k = 0; k < 3; ++k) cut_nh.push_back(m->n_hat[q * 3 + k]);
        }
      continue;
    }
    if (t[0] - 1 < 0 || t[0] - 1 >= m->ngrid) return fail(c, DSEM_ERR_INVALID_ARG, "mortar master id out of range");
    if (t[1] == 0) {  // boundary mortar: the master face's d%bcond selects the condition
      if (c->ncase != 1) return fail(c, DSEM_ERR_UNSUPPORTED, "boundary faces are not supported in an ensemble");
      if (!m->bcond) return fail(c, DSEM_ERR_INVALID_ARG, "boundary mortars (id(2)=0) need dsem_mesh_desc.bcond");
      const int id1 = t[0] - 1, f1 = t[2];
      if (f1 < 1 || f1 > 6) return fail(c, DSEM_ERR_INVALID_ARG, "bad mortar face or orientation");
      const int bc = m->bcond[6 * id1 + f1 - 1];
      if (bc < DSEM_BC_WALLADIAB || bc > DSEM_BC_OUTFLOW)
        return fail(c, DSEM_ERR_INVALID_ARG, "the master face of a boundary mortar has no boundary condition in bcond");
      const int G = ms.G(id1), G2 = G * G;
      if (t[4] != G || t[5] != G || t[8] != G || t[9] != G || t[10] != 0)
        return fail(c, DSEM_ERR_UNSUPPORTED, "boundary mortars must match their face's order, with orient 0");
      dsem::MortarB mb;
      mb.ms = c->groups[c->ext_group[id1]].f0 + (long long)c->ext_k[id1] * 30 * G2 + (long long)(f1 - 1) * 5 * G2;
      mb.geo = (int)bms[G].size();
      const bool low = (f1 == 1 || f1 == 3 || f1 == 6);
      mb.flags = bc | (low << 3) | ((t[12] < 0) << 4);
      bms[G].push_back(mb);
      bids[G].push_back(j);
      for (int jj = 0; jj < G; ++jj)
        for (int i = 0; i < G; ++i) {
          const size_t q = (size_t)j * ldx * ldx + i + (size_t)ldx * jj;
          bnrs[G].push_back(m->norm[q]);
          for (int k = 0; k < 3; ++k) bnhs[G].push_back(m->n_hat[q * 3 + k]);
        }
      if (bc == DSEM_BC_WALLISOTH) c->bnd_need_twall = true;
      if (bc == DSEM_BC_INFLOW || bc == DSEM_BC_OUTFLOW) c->bnd_need_ext = true;
      continue;
    }
    if (t[1] - 1 < 0) return fail(c, DSEM_ERR_INVALID_ARG, "mortar slave id out of range");
    if (t[1] - 1 >= m->ngrid) return fail(c, DSEM_ERR_INVALID_ARG, "mortar slave id out of range");
    const int id1 = t[0] - 1 + ms.el0[cs], id2 = t[1] - 1 + ms.el0[cs];
    const int f1 = t[2], f2 = t[3], orient = t[10];
    if (f1 < 1 || f1 > 6 || f2 < 1 || f2 > 6 || orient < 0 || orient > 7)
      return fail(c, DSEM_ERR_INVALID_ARG, "bad mortar face or orientation");
    const int Gm = ms.G(id1), Gs = ms.G(id2);
    const bool conf = t[13] && t[14] && t[15] && t[16];
    if (t[4] != Gm || t[5] != Gm || t[6] != Gs || t[7] != Gs || t[8] != std::max(Gm, Gs) || t[9] != std::max(Gm, Gs))
      return fail(c, DSEM_ERR_UNSUPPORTED, "mortar lengths must match the element orders (geometrically conforming faces)");
    if (!conf || Gm != Gs) {  // p-nonconforming mortar
      MortarNC nc{};
      const int G2m = Gm * Gm, G2s = Gs * Gs;
      nc.ms = c->groups[c->ext_group[id1]].f0 + (long long)c->ext_k[id1] * 30 * G2m + (long long)(f1 - 1) * 5 * G2m;
      nc.ss = c->groups[c->ext_group[id2]].f0 + (long long)c->ext_k[id2] * 30 * G2s + (long long)(f2 - 1) * 5 * G2s;
      nc.gm = Gm;
      nc.gs = Gs;
      nc.lm1 = t[8];
      nc.lm2 = t[9];
      nc.orient = orient;
      nc.sign = t[11];
      nc.nsign = t[12];
      nc.low = (f1 == 1 || f1 == 3 || f1 == 6);
      for (int k = 0; k < 4; ++k) nc.conf[k] = t[13 + k];
      nc.geo = (int)nc_nrm.size();
      for (int side = 0; side < 2; ++side)
        for (int dir = 0; dir < 2; ++dir) {
          nc.P[side][dir] = nc.R[side][dir] = -1;
          if (nc.conf[2 * side + dir]) continue;
          const int nin = side == 0 ? Gm : Gs, nout = t[8 + dir];
          const long long key = (long long)nin * 100 + nout;
          auto it = mat_off.find(key);
          if (it == mat_off.end()) {
            std::vector<double> ci(nin), co(nout), P((size_t)nout * nin), R((size_t)nin * nout);
            hostmath::gauss_points(nin, ci.data());
            hostmath::gauss_points(nout, co.data());
            hostmath::projection(ci.data(), nin, co.data(), nout, P.data());
            hostmath::projection(co.data(), nout, ci.data(), nin, R.data());
            const int po = (int)mats.size();
            mats.insert(mats.end(), P.begin(), P.end());
            const int ro = (int)mats.size();
            mats.insert(mats.end(), R.begin(), R.end());
            it = mat_off.emplace(key, std::make_pair(po, ro)).first;
          }
          nc.P[side][dir] = it->second.first;
          nc.R[side][dir] = it->second.second;
        }
      for (int jj = 0; jj < t[9]; ++jj)
        for (int i = 0; i < t[8]; ++i) {
          const size_t q = (size_t)j * ldx * ldx + i + (size_t)ldx * jj;
          nc_nrm.push_back(m->norm[q]);
          for (int k = 0; k < 3; ++k) nc_nh.push_back(m->n_hat[q * 3 + k]);
        }
      ncs.push_back(nc);
      continue;
    }
    const int G = Gm, G2 = G * G;
    const Group &gm = c->groups[c->ext_group[id1]];
    const Group &gs = c->groups[c->ext_group[id2]];
    MortarC mc;
    mc.ms = gm.f0 + (long long)c->ext_k[id1] * 30 * G2 + (long long)(f1 - 1) * 5 * G2;
    mc.ss = gs.f0 + (long long)c->ext_k[id2] * 30 * G2 + (long long)(f2 - 1) * 5 * G2;
    mc.geo = (int)mcs[G].size();
    const bool low = (f1 == 1 || f1 == 3 || f1 == 6);
    mc.flags = orient | ((t[11] < 0) << 3) | ((t[12] < 0) << 4) | (low << 5);
    mcs[G].push_back(mc);
    for (int jj = 0; jj < G; ++jj)
      for (int i = 0; i < G; ++i) {
        const size_t q = (size_t)j * ldx * ldx + i + (size_t)ldx * jj;
        nrs[G].push_back(m->norm[q]);
        for (int k = 0; k < 3; ++k) nhs[G].push_back(m->n_hat[q * 3 + k]);
      }
  }
  }  // cases
  for (int G = GMIN; G <= GMAX; ++G) {
    if (mcs[G].empty()) continue;
    MList ml;
    ml.G = G;
    ml.n = (int)mcs[G].size();
    CK(cudaMalloc(&ml.mc, mcs[G].size() * sizeof(MortarC)));
    CK(cudaMemcpy(ml.mc, mcs[G].data(), mcs[G].size() * sizeof(MortarC), cudaMemcpyHostToDevice));
    CK(cudaMalloc(&ml.nh, nhs[G].size() * sizeof(double)));
    CK(cudaMemcpy(ml.nh, nhs[G].data(), nhs[G].size() * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMalloc(&ml.nrm, nrs[G].size() * sizeof(double)));
    CK(cudaMemcpy(ml.nrm, nrs[G].data(), nrs[G].size() * sizeof(double), cudaMemcpyHostToDevice));
    c->mlists.push_back(ml);
  }
  for (int G = GMIN; G <= GMAX; ++G) {
    if (bms[G].empty()) continue;
    BList bl;
    bl.G = G;
    bl.n = (int)bms[G].size();
    bl.mortar = bids[G];
    const size_t next = (size_t)bl.n * 5 * G * G;
    CK(cudaMalloc(&bl.mb, bms[G].size() * sizeof(dsem::MortarB)));
    CK(cudaMemcpy(bl.mb, bms[G].data(), bms[G].size() * sizeof(dsem::MortarB), cudaMemcpyHostToDevice));
    CK(cudaMalloc(&bl.nh, bnhs[G].size() * sizeof(double)));
    CK(cudaMemcpy(bl.nh, bnhs[G].data(), bnhs[G].size() * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMalloc(&bl.nrm, bnrs[G].size() * sizeof(double)));
    CK(cudaMemcpy(bl.nrm, bnrs[G].data(), bnrs[G].size() * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMalloc(&bl.qext, next * sizeof(double)));
    CK(cudaMemset(bl.qext, 0, next * sizeof(double)));
    CK(cudaMalloc(&bl.fvext, next * sizeof(double)));
    CK(cudaMemset(bl.fvext, 0, next * sizeof(double)));
    c->nbnd += bl.n;
    c->blists.push_back(bl);
  }

  if (!cuts.empty()) {  // ghost g must appear on exactly one cut mortar
    const int n = (int)cuts.size();
    std::vector<long long> src(n, -1);
    for (int i = 0; i < n; ++i) {
      const int g = cut_ghost[i];
      if (g >= n || src[g] >= 0) return fail(c, DSEM_ERR_INVALID_ARG, "ghost faces must be numbered 1..ncut, each once");
      src[g] = cuts[i].ls;
    }
    c->ncut = n;
    c->cut_G = cut_G;
    CK(cudaMalloc(&c->cut, n * sizeof(MortarCut)));
    CK(cudaMemcpy(c->cut, cuts.data(), n * sizeof(MortarCut), cudaMemcpyHostToDevice));
    CK(cudaMalloc(&c->cut_nh, cut_nh.size() * sizeof(double)));
    CK(cudaMemcpy(c->cut_nh, cut_nh.data(), cut_nh.size() * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMalloc(&c->cut_nrm, cut_nrm.size() * sizeof(double)));
    CK(cudaMemcpy(c->cut_nrm, cut_nrm.data(), cut_nrm.size() * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMalloc(&c->pack_src, n * sizeof(long long)));
    CK(cudaMemcpy(c->pack_src, src.data(), n * sizeof(long long), cudaMemcpyHostToDevice));
    const size_t nb = (size_t)n * 5 * cut_G * cut_G * sizeof(double);
    CK(cudaMalloc(&c->send, nb));
    CK(cudaMalloc(&c->ghost, nb));
    CK(cudaMemset(c->send, 0, nb));
    CK(cudaMemset(c->ghost, 0, nb));
  }

  if (!ncs.empty()) {
    c->nnc = (int)ncs.size();
    CK(cudaMalloc(&c->nc, ncs.size() * sizeof(MortarNC)));
    CK(cudaMemcpy(c->nc, ncs.data(), ncs.size() * sizeof(MortarNC), cudaMemcpyHostToDevice));
    CK(cudaMalloc(&c->nc_nh, nc_nh.size() * sizeof(double)));
    CK(cudaMemcpy(c->nc_nh, nc_nh.data(), nc_nh.size() * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMalloc(&c->nc_nrm, nc_nrm.size() * sizeof(double)));
    CK(cudaMemcpy(c->nc_nrm, nc_nrm.data(), nc_nrm.size() * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMalloc(&c->nc_mats, std::max<size_t>(1, mats.size()) * sizeof(double)));
    if (!mats.empty()) CK(cudaMemcpy(c->nc_mats, mats.data(), mats.size() * sizeof(double), cudaMemcpyHostToDevice));
  }

  // the mortar of each element face, for the update kernel that averages the viscous face
  // fluxes itself (dsem_step): only when every face is one side of exactly one conforming
  // mortar (no boundary, p-nonconforming or cut faces)
  if (ncs.empty() && cuts.empty() && c->blists.empty() && !c->groups.empty()) {
    const size_t ng = c->groups.size();
    std::vector<std::vector<MortarC>> fm(ng);
    std::vector<std::vector<char>> seen(ng);
    for (size_t gi = 0; gi < ng; ++gi) {
      fm[gi].resize(6 * (size_t)c->groups[gi].nel);
      seen[gi].assign(6 * (size_t)c->groups[gi].nel, 0);
    }
    bool ok = true;
    for (int G = GMIN; G <= GMAX && ok; ++G)
      for (const MortarC &m : mcs[G]) {
        const long long G2 = (long long)G * G;
        for (int side = 0; side < 2 && ok; ++side) {
          const long long off = side ? m.ss : m.ms;
          ok = false;
          for (size_t gi = 0; gi < ng; ++gi) {
            const Group &g = c->groups[gi];
            if (g.G != G || off < g.f0 || off >= g.f0 + (long long)g.nel * 30 * G2) continue;
            const long long rel = off - g.f0, slot = rel / (5 * G2);
            if (rel % (5 * G2) != 0 || seen[gi][slot]) break;
            seen[gi][slot] = 1;
            MortarC e = m;
            e.flags |= side << 8;
            fm[gi][slot] = e;
            ok = true;
            break;
          }
        }
        if (!ok) break;
      }
    for (size_t gi = 0; gi < ng && ok; ++gi)
      for (char s : seen[gi]) ok = ok && s;
    if (ok) {
      for (size_t gi = 0; gi < ng; ++gi) {
        Group &g = c->groups[gi];
        CK(cudaMalloc(&g.fmc, fm[gi].size() * sizeof(MortarC)));
        CK(cudaMemcpy(g.fmc, fm[gi].data(), fm[gi].size() * sizeof(MortarC), cudaMemcpyHostToDevice));
      }
      c->fuse_vis = true;
    }
  }

  // ---- state and face buffers
  CK(cudaMalloc(&c->JQ, c->nq * sizeof(double)));
  CK(cudaMalloc(&c->gQ, c->nq * sizeof(double)));
  CK(cudaMalloc(&c->QTI, c->nq * sizeof(double)));
  CK(cudaMalloc(&c->Qt, c->nq * sizeof(double)));
  CK(cudaMemset(c->JQ, 0, c->nq * sizeof(double)));
  CK(cudaMemset(c->gQ, 0, c->nq * sizeof(double)));
  CK(cudaMalloc(&c->QF, c->nface * sizeof(double)));
  CK(cudaMalloc(&c->FF, c->nface * sizeof(double)));
  CK(cudaMalloc(&c->VF, c->nface * sizeof(double)));
  CK(cudaMalloc(&c->part, (size_t)ngrid * 5 * sizeof(double)));
  CK(cudaMalloc(&c->flag, sizeof(int)));
  CK(cudaMemset(c->flag, 0, sizeof(int)));
  CK(cudaEventCreate(&c->e0));
  CK(cudaEventCreate(&c->e1));
  // per-case tables
  {
    std::vector<double> rec(2 * (size_t)c->ncase);
    for (int k = 0; k < c->ncase; ++k) {
      rec[2 * k] = c->case_re[k];
      rec[2 * k + 1] = 1.0 / c->case_re[k];
    }
    CK(cudaMalloc(&c->d_rec, rec.size() * sizeof(double)));
    CK(cudaMemcpy(c->d_rec, rec.data(), rec.size() * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMalloc(&c->d_dtc, (size_t)c->ncase * sizeof(double)));
    CK(cudaMemset(c->d_dtc, 0, (size_t)c->ncase * sizeof(double)));
  }
  // streams for the parallel branches of a stage
  {
    const size_t nj = std::max(c->groups.size(), c->mlists.size() + (c->nnc > 0 ? 1 : 0) + c->blists.size());
    if (nj > 1) {
      CK(cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming));
      for (size_t j = 0; j < nj; ++j) {
        cudaStream_t s;
        cudaEvent_t e;
        CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        c->aux.push_back(s);
        CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        c->ev_join.push_back(e);
      }
    }
  }
  // set the shared-memory attribute of every volume variant outside any capture
  for (auto &g : c->groups)
    for (int mode = 0; mode < 4; ++mode) {
      VolArgs a{};
      CK(with_G(g.G, [&](auto gg) { return Launch<decltype(gg)::value>::vol(a, 0, g.diag, mode, c->st); }));
    }
  return DSEM_OK;
}

}  // namespace

extern "C" {

void dsem_destroy(dsem_ctx *c) {
  if (!c) return;
  if (c->gexec) cudaGraphExecDestroy(c->gexec);
  for (auto &g : c->groups) {
    cudaFree(g.jac);
    cudaFree(g.gg);
    cudaFree(g.gm);
    cudaFree(g.hd);
    cudaFree(g.muhg);
    cudaFree(g.EVB);
    cudaFree(g.kew);
    cudaFree(g.int2ext);
    cudaFree(g.ecase);
    cudaFree(g.nuhg);
    cudaFree(g.sens);
    cudaFree(g.fmc);
  }
  cudaFree(c->d_rec);
  cudaFree(c->d_dtc);
  cudaFree(c->cut);
  cudaFree(c->cut_nh);
  cudaFree(c->cut_nrm);
  cudaFree(c->pack_src);
  cudaFree(c->send);
  cudaFree(c->ghost);
  for (auto s : c->aux) cudaStreamDestroy(s);
  for (auto e : c->ev_join) cudaEventDestroy(e);
  if (c->ev_fork) cudaEventDestroy(c->ev_fork);
  cudaFree(c->nc);
  cudaFree(c->nc_nh);
  cudaFree(c->nc_nrm);
  cudaFree(c->nc_mats);
  for (auto &ml : c->mlists) {
    cudaFree(ml.mc);
    cudaFree(ml.nh);
    cudaFree(ml.nrm);
  }
  for (auto &bl : c->blists) {
    cudaFree(bl.mb);
    cudaFree(bl.nh);
    cudaFree(bl.nrm);
    cudaFree(bl.qext);
    cudaFree(bl.fvext);
  }
  cudaFree(c->QLB);
  cudaFree(c->JQ);
  cudaFree(c->gQ);
  cudaFree(c->QTI);
  cudaFree(c->Qt);
  cudaFree(c->QF);
  cudaFree(c->FF);
  cudaFree(c->VF);
  cudaFree(c->stage);
  cudaFree(c->part);
  cudaFree(c->flag);
  if (c->e0) cudaEventDestroy(c->e0);
  if (c->e1) cudaEventDestroy(c->e1);
  if (c->st) cudaStreamDestroy(c->st);
  delete c;
}

int dsem_upload_q(dsem_ctx *c, const double *JQ, int ldx) {
  if (!c || !JQ) return fail(c, DSEM_ERR_INVALID_ARG, "null argument");
  int r = check_ldx(c, ldx);
  if (r) return r;
  r = ensure_stage_buf(c, ldx, 5);
  if (r) return r;
  const size_t n = (size_t)c->ngrid * 5 * ldx * ldx * ldx;
  CK(cudaMemcpyAsync(c->stage, JQ, n * sizeof(double), cudaMemcpyHostToDevice, c->st));
  for (auto &g : c->groups) {
    k_pack<<<g.nel, 256, 0, c->st>>>(c->stage, ldx, g.int2ext, 0, g.G, 5, c->JQ + g.q0, 1);
    CK(cudaGetLastError());
  }
  long long l = 0;
  r = enqueue_traces(c, &l);
  if (r) return r;
  CK(cudaStreamSynchronize(c->st));
  return DSEM_OK;
}

int dsem_download_q(dsem_ctx *c, double *JQ, int ldx) {
  if (!c || !JQ) return fail(c, DSEM_ERR_INVALID_ARG, "null argument");
  int r = check_ldx(c, ldx);
  if (r) return r;
  return unpack_to_host(c, c->JQ, JQ, ldx, 5, state_offs(c));
}

int dsem_rhs(dsem_ctx *c, double tk, double *Qt, int ldx) {
  (void)tk;
  if (!c) return fail(c, DSEM_ERR_INVALID_ARG, "null context");
  if (c->ncut) return fail(c, DSEM_ERR_INVALID_ARG, "a shard advances with dsem_shard_stage");
  if (Qt) {
    int r = check_ldx(c, ldx);
    if (r) return r;
  }
  long long l = 0;
  int r;
  if (!c->traces_valid && (r = enqueue_traces(c, &l))) return r;
  CK(cudaMemsetAsync(c->flag, 0, sizeof(int), c->st));
  r = enqueue_stage(c, 0, true, c->Qt, &l);
  if (r) return r;
  c->grad_valid = true;
  c->ev_grad_valid = c->shock != 0;
  if (Qt && (r = unpack_to_host(c, c->Qt, Qt, ldx, 5, state_offs(c)))) return r;
  return check_flag(c);
}

}  // extern "C"

namespace {
// dt of every case for the stages enqueued next (read by k_update)
int set_dt(dsem_ctx *c, const double *dt) {
  for (int k = 0; k < c->ncase; ++k) {
    if (!std::isfinite(dt[k])) return fail(c, DSEM_ERR_INVALID_ARG, "dt is not finite");
    c->case_dt[k] = dt[k];
  }
  CK(cudaMemcpyAsync(c->d_dtc, c->case_dt.data(), (size_t)c->ncase * sizeof(double), cudaMemcpyHostToDevice, c->st));
  return DSEM_OK;
}

int step_impl(dsem_ctx *c, int nsteps) {
  const int nsteps0 = nsteps;
  long long l = 0;
  int r;
  if (!c->traces_valid && (r = enqueue_traces(c, &l))) return r;
  CK(cudaMemsetAsync(c->flag, 0, sizeof(int), c->st));
  const bool save = c->shock || c->keep_grad || c->les;
  long long per_step = 0;
  // the first step of a run may need EV / LES without valid gradients: run it eagerly
  CK(cudaEventRecord(c->e0, c->st));
  if (nsteps > 0 && ((c->shock && !c->ev_grad_valid) || (c->les && !c->grad_valid))) {
    if ((r = enqueue_step(c, save, &per_step))) return r;
    c->ev_grad_valid = true;
    c->grad_valid = true;
    --nsteps;
  }
  long long launches = per_step;
  if (nsteps > 0) {
    const int key = (save ? 1 : 0) | (c->ev_grad_valid ? 2 : 0) | (c->grad_valid ? 4 : 0) | (c->les ? 8 : 0) |
                    (c->keep_lob ? 16 : 0);
    if (!c->gexec || c->graph_key != key) {
      if (c->gexec) cudaGraphExecDestroy(c->gexec);
      c->gexec = nullptr;
      cudaGraph_t graph;
      CK(cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal));
      long long cnt = 0;
      r = enqueue_step(c, save, &cnt);
      cudaError_t ec = cudaStreamEndCapture(c->st, &graph);
      if (r) return r;
      if (ec != cudaSuccess) return cuda_fail(c, ec, "cudaStreamEndCapture");
      ec = cudaGraphInstantiate(&c->gexec, graph, 0);
      cudaGraphDestroy(graph);
      if (ec != cudaSuccess) return cuda_fail(c, ec, "cudaGraphInstantiate");
      c->graph_key = key;
      c->graph_launches = cnt;
    }
    for (int s = 0; s < nsteps; ++s) CK(cudaGraphLaunch(c->gexec, c->st));
    launches += c->graph_launches * nsteps;
    c->grad_valid = c->grad_valid || save;
    c->ev_grad_valid = c->ev_grad_valid || c->shock;
  }
  CK(cudaEventRecord(c->e1, c->st));
  CK(cudaEventSynchronize(c->e1));
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, c->e0, c->e1));
  c->last_ms = ms;
  c->last_launches = launches;
  if (save) c->grad_valid = true;
  if (c->keep_lob && nsteps0 > 0) c->lob_valid = true;
  return check_flag(c);
}

// KE, -dKE/dt and the enstrophy dissipation of every case
int diag_impl(dsem_ctx *c, const double *dt, int first, double *ke, double *dkdt, double *eps) {
  c->keep_grad = 1;
  const bool have = c->grad_valid;
  for (auto &g : c->groups) {
    k_diag<<<g.nel, 128, sizeof(double) * 5 * g.G * g.G * g.G, c->st>>>(c->JQ + g.q0, g.jac, g.EVB, g.kew, g.G, g.nel,
                                                                         have ? 1 : 0, c->part + g.e0 * 5);
    CK(cudaGetLastError());
  }
  c->host_part.resize((size_t)c->ngrid * 5);
  CK(cudaMemcpyAsync(c->host_part.data(), c->part, c->host_part.size() * sizeof(double), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  const double PI = hostmath::PI;
  for (int k = 0; k < c->ncase; ++k) {
    double us = 0, vs = 0, ws = 0, s = 0, s2 = 0;
    for (int e = c->case_el0[k]; e < c->case_el0[k + 1]; ++e) {  // caller element order
      const auto &g = c->groups[c->ext_group[e]];
      const double *p = &c->host_part[(size_t)(g.e0 + c->ext_k[e]) * 5];
      us += p[0];
      vs += p[1];
      ws += p[2];
      s += p[3];
      s2 += p[4];
    }
    // jacob(1,1,1) of the case's element 1
    double j0 = 0.0;
    {
      const int e1 = c->case_el0[k];
      const auto &g = c->groups[c->ext_group[e1]];
      CK(cudaMemcpy(&j0, g.jac + (size_t)c->ext_k[e1] * g.G * g.G * g.G, sizeof(double), cudaMemcpyDeviceToHost));
    }
    us /= j0;
    vs /= j0;
    ws /= j0;
    const double tk = 0.5 * (us + vs + ws) / (8.0 * PI * PI * PI);
    if (first) c->case_prestep[k] = 0.0;
    if (ke) ke[k] = tk;
    if (dkdt) dkdt[k] = (c->case_prestep[k] - tk) / dt[k];
    c->case_prestep[k] = tk;
    if (eps) eps[k] = (have && s2 > 0) ? 100.0 * (s / s2) * (1.0 / c->case_re[k]) : 0.0;
  }
  return DSEM_OK;
}

int check_case(dsem_ctx *c, int k) {
  if (k < 0 || k >= c->ncase) return fail(c, DSEM_ERR_INVALID_ARG, "case index out of range");
  return DSEM_OK;
}
}  // namespace

extern "C" {

int dsem_stage(dsem_ctx *c, double time, double dt, int kk, double *Qt, int ldx) {
  (void)time;
  if (!c) return fail(c, DSEM_ERR_INVALID_ARG, "null context");
  if (c->ncut) return fail(c, DSEM_ERR_INVALID_ARG, "a shard advances with dsem_shard_stage");
  if (kk < 1 || kk > c->kord) return fail(c, DSEM_ERR_INVALID_ARG, "stage index outside 1..kord");
  if (Qt) {
    int r = check_ldx(c, ldx);
    if (r) return r;
  }
  std::vector<double> dts(c->ncase, dt);
  int r = set_dt(c, dts.data());
  if (r) return r;
  long long l = 0;
  if (!c->traces_valid && (r = enqueue_traces(c, &l))) return r;
  CK(cudaMemsetAsync(c->flag, 0, sizeof(int), c->st));
  if (kk == 1 && c->shock && (r = enqueue_ev(c, &l))) return r;
  if (kk == 1 && c->les && (r = enqueue_les(c, &l))) return r;
  r = enqueue_stage(c, kk, true, Qt ? c->Qt : nullptr, &l);
  if (r) return r;
  c->grad_valid = true;
  c->ev_grad_valid = c->shock != 0;
  if (kk == c->kord && c->keep_lob) c->lob_valid = true;
  if (Qt && (r = unpack_to_host(c, c->Qt, Qt, ldx, 5, state_offs(c)))) return r;
  return check_flag(c);
}

int dsem_keep_lobatto(dsem_ctx *c, int on) {
  if (!c) return fail(c, DSEM_ERR_INVALID_ARG, "null context");
  if (c->ncut) return fail(c, DSEM_ERR_UNSUPPORTED, "sharded contexts do not keep Lobatto arrays");
  if (on && !c->QLB) {
    long long n = 0;
    for (auto &g : c->groups) {
      g.l0 = n;
      n += (long long)g.nel * 15 * (g.G + 1) * g.G * g.G;
    }
    CK(cudaMalloc(&c->QLB, (size_t)std::max(n, 1LL) * sizeof(double)));
  }
  c->keep_lob = on != 0;
  c->lob_valid = false;
  return DSEM_OK;
}

int dsem_step(dsem_ctx *c, double time, double dt, int nsteps) {
  (void)time;
  if (!c) return fail(c, DSEM_ERR_INVALID_ARG, "null context");
  if (c->ncut) return fail(c, DSEM_ERR_INVALID_ARG, "a shard advances with dsem_shard_stage");
  if (nsteps < 0) return fail(c, DSEM_ERR_INVALID_ARG, "negative step count");
  std::vector<double> dts(c->ncase, dt);
  const int r = set_dt(c, dts.data());
  if (r) return r;
  return step_impl(c, nsteps);
}

int dsem_step_batch(dsem_ctx *c, const double *dt, int nsteps) {
  if (!c || !dt) return fail(c, DSEM_ERR_INVALID_ARG, "null argument");
  if (c->ncut) return fail(c, DSEM_ERR_INVALID_ARG, "a shard advances with dsem_shard_stage");
  if (nsteps < 0) return fail(c, DSEM_ERR_INVALID_ARG, "negative step count");
  const int r = set_dt(c, dt);
  if (r) return r;
  return step_impl(c, nsteps);
}

int dsem_diag(dsem_ctx *c, double dt, int first, double *ke, double *dkdt, double *eps) {
  if (!c) return fail(c, DSEM_ERR_INVALID_ARG, "null context");
  if (c->ncase != 1) return fail(c, DSEM_ERR_INVALID_ARG, "a batch reports per case: use dsem_diag_batch");
  return diag_impl(c, &dt, first, ke, dkdt, eps);
}

int dsem_diag_batch(dsem_ctx *c, const double *dt, int first, double *ke, double *dkdt, double *eps) {
  if (!c || !dt) return fail(c, DSEM_ERR_INVALID_ARG, "null argument");
  return diag_impl(c, dt, first, ke, dkdt, eps);
}

int dsem_batch_size(const dsem_ctx *c) { return c ? c->ncase : DSEM_ERR_INVALID_ARG; }

int dsem_upload_q_case(dsem_ctx *c, int k, const double *JQ, int ldx) {
  if (!c || !JQ) return fail(c, DSEM_ERR_INVALID_ARG, "null argument");
  int r = check_case(c, k);
  if (r) return r;
  for (auto &g : c->groups)
    if (g.case_hi[k] > g.case_lo[k] && ldx < g.G) return fail(c, DSEM_ERR_INVALID_ARG, "ldx smaller than the number of Gauss points");
  if ((r = ensure_stage_buf(c, ldx, 5))) return r;
  const size_t n = (size_t)(c->case_el0[k + 1] - c->case_el0[k]) * 5 * ldx * ldx * ldx;
  CK(cudaMemcpyAsync(c->stage, JQ, n * sizeof(double), cudaMemcpyHostToDevice, c->st));
  for (auto &g : c->groups) {
    const int lo = g.case_lo[k], nk = g.case_hi[k] - lo;
    if (nk <= 0) continue;
    k_pack<<<nk, 256, 0, c->st>>>(c->stage, ldx, g.int2ext + lo, c->case_el0[k], g.G, 5,
                                  c->JQ + g.q0 + (long long)lo * 5 * g.G * g.G * g.G, 1);
    CK(cudaGetLastError());
  }
  long long l = 0;
  if ((r = enqueue_traces(c, &l))) return r;
  CK(cudaStreamSynchronize(c->st));
  return DSEM_OK;
}

int dsem_download_q_case(dsem_ctx *c, int k, double *JQ, int ldx) {
  if (!c || !JQ) return fail(c, DSEM_ERR_INVALID_ARG, "null argument");
  int r = check_case(c, k);
  if (r) return r;
  for (auto &g : c->groups)
    if (g.case_hi[k] > g.case_lo[k] && ldx < g.G) return fail(c, DSEM_ERR_INVALID_ARG, "ldx smaller than the number of Gauss points");
  if ((r = ensure_stage_buf(c, ldx, 5))) return r;
  const size_t n = (size_t)(c->case_el0[k + 1] - c->case_el0[k]) * 5 * ldx * ldx * ldx;
  CK(cudaMemsetAsync(c->stage, 0, n * sizeof(double), c->st));
  for (auto &g : c->groups) {
    const int lo = g.case_lo[k], nk = g.case_hi[k] - lo;
    if (nk <= 0) continue;
    k_pack<<<nk, 256, 0, c->st>>>(c->JQ + g.q0 + (long long)lo * 5 * g.G * g.G * g.G, ldx, g.int2ext + lo,
                                  c->case_el0[k], g.G, 5, c->stage, 0);
    CK(cudaGetLastError());
  }
  CK(cudaMemcpyAsync(JQ, c->stage, n * sizeof(double), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return DSEM_OK;
}

int dsem_get_muhg(dsem_ctx *c, double *mu, int ldx) {
  if (!c || !mu) return fail(c, DSEM_ERR_INVALID_ARG, "null argument");
  int r = check_ldx(c, ldx);
  if (r) return r;
  std::vector<long long> offs;
  // muhg lives in per-group arrays: unpack group by group
  r = ensure_stage_buf(c, ldx, 1);
  if (r) return r;
  const size_t n = (size_t)c->ngrid * ldx * ldx * ldx;
  CK(cudaMemsetAsync(c->stage, 0, n * sizeof(double), c->st));
  for (auto &g : c->groups) {
    k_pack<<<g.nel, 256, 0, c->st>>>(g.muhg, ldx, g.int2ext, 0, g.G, 1, c->stage, 0);
    CK(cudaGetLastError());
  }
  CK(cudaMemcpyAsync(mu, c->stage, n * sizeof(double), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return DSEM_OK;
}

int dsem_shard_info(const dsem_ctx *c, int *nghost, int *doubles_per_face, double **send, double **ghost) {
  if (!c) return DSEM_ERR_INVALID_ARG;
  if (nghost) *nghost = c->ncut;
  if (doubles_per_face) *doubles_per_face = 5 * c->cut_G * c->cut_G;
  if (send) *send = c->send;
  if (ghost) *ghost = c->ghost;
  return DSEM_OK;
}

namespace {
// Enqueues one phase of a sharded stage on the context's stream (no wait).
int shard_enqueue(dsem_ctx *c, double dt, int kk, int phase) {
  if (!c) return fail(c, DSEM_ERR_INVALID_ARG, "null context");
  if (kk < 1 || kk > c->kord || phase < 0 || phase > 2)
    return fail(c, DSEM_ERR_INVALID_ARG, "stage index outside 1..kord or phase outside 0..2");
  long long l = 0;
  int r;
  const unsigned nb = (unsigned)std::min<long long>(((long long)c->ncut * 5 * c->cut_G * c->cut_G + 255) / 256, 148LL * 8);
  if (phase == 0) {  // stage start; local cut-face traces -> send
    if (!c->traces_valid && (r = enqueue_traces(c, &l))) return r;
    if (kk == 1) {
      CK(cudaMemsetAsync(c->flag, 0, sizeof(int), c->st));
      if (c->shock && (r = enqueue_ev(c, &l))) return r;
      if (c->les && (r = enqueue_les(c, &l))) return r;
    }
    std::vector<double> dts(c->ncase, dt);
    if ((r = set_dt(c, dts.data()))) return r;
    if (c->ncut) {
      k_pack_cut<<<std::max(nb, 1u), 256, 0, c->st>>>(c->pack_src, c->ncut, 5 * c->cut_G * c->cut_G, c->QF, c->send);
      CK(cudaGetLastError());
    }
  } else if (phase == 1) {  // ghost traces in; inviscid mortars, volume; local cut-face VF -> send
    const bool save = kk == c->kord && (c->shock || c->keep_grad || c->les);
    if ((r = enqueue_face_inv(c, &l)) || (r = enqueue_vol(c, save, &l))) return r;
    if (c->ncut) {
      k_pack_cut<<<std::max(nb, 1u), 256, 0, c->st>>>(c->pack_src, c->ncut, 5 * c->cut_G * c->cut_G, c->VF, c->send);
      CK(cudaGetLastError());
    }
  } else {  // ghost VF in; viscous mortars, update
    if ((r = enqueue_face_vis(c, &l)) || (r = enqueue_update(c, kk, nullptr, &l))) return r;
    if (kk == c->kord) {
      const bool save = c->shock || c->keep_grad || c->les;
      c->grad_valid = c->grad_valid || save;
      c->ev_grad_valid = c->ev_grad_valid || c->shock;
    }
  }
  return DSEM_OK;
}
}  // namespace

int dsem_shard_stage(dsem_ctx *c, double dt, int kk, int phase) {
  int r = shard_enqueue(c, dt, kk, phase);
  if (r) return r;
  if (phase == 2 && kk == c->kord) return check_flag(c);
  CK(cudaStreamSynchronize(c->st));
  return DSEM_OK;
}

int dsem_shard_enqueue(dsem_ctx *c, double dt, int kk, int phase) { return shard_enqueue(c, dt, kk, phase); }

int dsem_shard_finish(dsem_ctx *c) {
  if (!c) return fail(c, DSEM_ERR_INVALID_ARG, "null context");
  return check_flag(c);
}

int dsem_get_stream(const dsem_ctx *c, void **stream) {
  if (!c || !stream) return DSEM_ERR_INVALID_ARG;
  *stream = static_cast<void *>(c->st);
  return DSEM_OK;
}

int dsem_diag_sums(dsem_ctx *c, double *sums) {
  if (!c || !sums) return fail(c, DSEM_ERR_INVALID_ARG, "null argument");
  c->keep_grad = 1;
  const bool have = c->grad_valid;
  for (auto &g : c->groups) {
    k_diag<<<g.nel, 128, sizeof(double) * 5 * g.G * g.G * g.G, c->st>>>(c->JQ + g.q0, g.jac, g.EVB, g.kew, g.G, g.nel,
                                                                         have ? 1 : 0, c->part + g.e0 * 5);
    CK(cudaGetLastError());
  }
  c->host_part.resize((size_t)c->ngrid * 5);
  CK(cudaMemcpyAsync(c->host_part.data(), c->part, c->host_part.size() * sizeof(double), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  for (int k = 0; k < 5; ++k) sums[k] = 0.0;
  for (int e = 0; e < c->ngrid; ++e) {
    const auto &g = c->groups[c->ext_group[e]];
    const double *p = &c->host_part[(size_t)(g.e0 + c->ext_k[e]) * 5];
    for (int k = 0; k < 5; ++k) sums[k] += p[k];
  }
  const auto &g = c->groups[c->ext_group[0]];
  CK(cudaMemcpy(&sums[5], g.jac + (size_t)c->ext_k[0] * g.G * g.G * g.G, sizeof(double), cudaMemcpyDeviceToHost));
  sums[6] = have ? 1.0 : 0.0;
  return DSEM_OK;
}

int dsem_set_boundary(dsem_ctx *c, double twall, const double *Qext, const double *fvext, int ldx) {
  if (!c) return fail(c, DSEM_ERR_INVALID_ARG, "null context");
  if (!std::isfinite(twall)) return fail(c, DSEM_ERR_INVALID_ARG, "twall is not finite");
  if ((Qext || fvext) && !c->nbnd) return fail(c, DSEM_ERR_INVALID_ARG, "the mesh has no boundary faces");
  for (auto &bl : c->blists)
    if ((Qext || fvext) && ldx < bl.G) return fail(c, DSEM_ERR_INVALID_ARG, "ldx smaller than the number of Gauss points");
  if (twall != c->twall && c->gexec) {  // twall is a kernel parameter of the captured step
    cudaGraphExecDestroy(c->gexec);
    c->gexec = nullptr;
  }
  c->twall = twall;
  c->bnd_twall_set = true;
  // caller layout [nmort][5][ldx][ldx] (mrtr(:)%Q(:,:,:,2), i fastest) -> [entry][5][G^2]
  for (auto &bl : c->blists) {
    const int G = bl.G, G2 = G * G;
    std::vector<double> h((size_t)bl.n * 5 * G2);
    for (int which = 0; which < 2; ++which) {
      const double *src = which ? fvext : Qext;
      if (!src) continue;
      for (int k = 0; k < bl.n; ++k)
        for (int v = 0; v < 5; ++v)
          for (int j = 0; j < G; ++j)
            for (int i = 0; i < G; ++i)
              h[((size_t)k * 5 + v) * G2 + i + G * j] =
                  src[((((size_t)bl.mortar[k] * 5 + v) * ldx + j) * ldx) + i];
      CK(cudaMemcpyAsync(which ? bl.fvext : bl.qext, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice,
                         c->st));
      CK(cudaStreamSynchronize(c->st));
    }
  }
  if (Qext) c->bnd_ext_set = true;
  return DSEM_OK;
}

// Chooses, per element order, the launch shape of the volume kernel (threads
// per element and elements per SM) by timing the available shapes on the
// context's own elements and state.  All shapes give identical results.
int dsem_autotune(dsem_ctx *c, int reps, int *choice, double *ms) {
  static_assert(DSEM_VOL_VARIANTS == dsem::VOL_VARIANTS, "variant count");
  if (!c || reps < 1) return fail(c, DSEM_ERR_INVALID_ARG, "null context or reps < 1");
  long long l = 0;
  int r;
  if (!c->traces_valid && (r = enqueue_traces(c, &l))) return r;
  if (ms)
    for (int i = 0; i < DSEM_MAX_ORDER * DSEM_VOL_VARIANTS; ++i) ms[i] = -1.0;
  const int mode = vol_mode(c, false);
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  for (auto &g : c->groups) {
    const int slot = g.G - 2;  // order p = G - 1 at index p - 1
    int nv = 1;
    CK(with_G(g.G, [&](auto gg) {
      nv = Launch<decltype(gg)::value>::vol_variants();
      return cudaSuccess;
    }));
    if (!g.diag || mode == VOL_EV || mode == VOL_EV_SAVE) nv = 1;  // shapes exist for the plain diagonal kernel
    const VolArgs a = vol_args(c, g);
    int best = 0;
    float tbest = 0.f;
    for (int v = 0; v < nv; ++v) {
      auto launch = [&]() {
        return with_G(g.G, [&](auto gg) { return Launch<decltype(gg)::value>::vol(a, g.nel, true, mode, c->st, v); });
      };
      CK(launch());  // warm-up (and the kernel's one-time attributes)
      CK(cudaEventRecord(e0, c->st));
      for (int i = 0; i < reps; ++i) CK(launch());
      CK(cudaEventRecord(e1, c->st));
      CK(cudaEventSynchronize(e1));
      float t = 0.f;
      CK(cudaEventElapsedTime(&t, e0, e1));
      t /= (float)reps;
      if (ms) ms[slot * DSEM_VOL_VARIANTS + v] = t;
      if (v == 0 || t < tbest) {
        tbest = t;
        best = v;
      }
    }
    c->vol_variant[g.G] = best;
    if (choice) choice[slot] = best;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (c->gexec) {  // the captured step holds the old launch shapes
    cudaGraphExecDestroy(c->gexec);
    c->gexec = nullptr;
  }
  return DSEM_OK;
}

int dsem_set_vol_variant(dsem_ctx *c, int p, int variant) {
  if (!c || p < 1 || p > DSEM_MAX_ORDER) return fail(c, DSEM_ERR_INVALID_ARG, "null context or order outside 1..8");
  int nv = 1;
  CK(with_G(p + 1, [&](auto gg) {
    nv = Launch<decltype(gg)::value>::vol_variants();
    return cudaSuccess;
  }));
  if (variant < 0 || variant >= nv) return fail(c, DSEM_ERR_INVALID_ARG, "no such launch shape for this order");
  c->vol_variant[p + 1] = variant;
  if (c->gexec) {
    cudaGraphExecDestroy(c->gexec);
    c->gexec = nullptr;
  }
  return DSEM_OK;
}

int dsem_set_les(dsem_ctx *c, double cs, double numax) {
  if (!c) return fail(c, DSEM_ERR_INVALID_ARG, "null context");
  if (!(cs >= 0.0) || !(numax >= 0.0)) return fail(c, DSEM_ERR_INVALID_ARG, "cs and numax must be >= 0");
  if (cs > 0.0) {
    for (auto &g : c->groups)
      if (!g.diag) return fail(c, DSEM_ERR_UNSUPPORTED, "LES needs axis-aligned (diagonal-metric) elements");
    for (auto &g : c->groups) {
      if (!g.nuhg) {
        const size_t n = (size_t)g.nel * g.G * g.G * g.G;
        CK(cudaMalloc(&g.nuhg, n * sizeof(double)));
        CK(cudaMemset(g.nuhg, 0, n * sizeof(double)));
      }
    }
  }
  c->les = cs > 0.0 ? 1 : 0;
  c->les_cs = cs;
  c->les_numax = numax;
  if (c->gexec) {  // the captured step changes
    cudaGraphExecDestroy(c->gexec);
    c->gexec = nullptr;
  }
  return DSEM_OK;
}

int dsem_set_les_sensors(dsem_ctx *c, int shock_sensor, int rho_sensor) {
  if (!c) return fail(c, DSEM_ERR_INVALID_ARG, "null context");
  const int f = (shock_sensor ? 1 : 0) | (rho_sensor ? 2 : 0);
  if (f) {
    for (auto &g : c->groups) {
      if (!g.sens) {
        const size_t n = (size_t)g.nel * 2 * g.G * g.G * g.G;
        CK(cudaMalloc(&g.sens, n * sizeof(double)));
        CK(cudaMemset(g.sens, 0, n * sizeof(double)));
      }
    }
  }
  c->les_sensors = f;
  if (c->gexec) {  // the captured step changes
    cudaGraphExecDestroy(c->gexec);
    c->gexec = nullptr;
  }
  return DSEM_OK;
}

int dsem_get_nut(dsem_ctx *c, double *nu, int ldx) {
  if (!c || !nu) return fail(c, DSEM_ERR_INVALID_ARG, "null argument");
  if (!c->les) return fail(c, DSEM_ERR_INVALID_ARG, "LES is off (dsem_set_les)");
  int r = check_ldx(c, ldx);
  if (r) return r;
  r = ensure_stage_buf(c, ldx, 1);
  if (r) return r;
  const size_t n = (size_t)c->ngrid * ldx * ldx * ldx;
  CK(cudaMemsetAsync(c->stage, 0, n * sizeof(double), c->st));
  for (auto &g : c->groups) {
    k_pack<<<g.nel, 256, 0, c->st>>>(g.nuhg, ldx, g.int2ext, 0, g.G, 1, c->stage, 0);
    CK(cudaGetLastError());
  }
  CK(cudaMemcpyAsync(nu, c->stage, n * sizeof(double), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return DSEM_OK;
}

}  // extern "C"

namespace {
// Snapshot layout: header, then JQ (internal order), then the saved gradients
// of every group when they are valid.  The header pins the mesh layout.
struct StateHeader {
  char magic[8];
  long long version, ngrid, nmort, ncase, ngroups, nq, nevb, flags;
  long long layout;  // hash of the groups' (order, element count)
  double prestep[1];  // ncase values follow in the blob (prestep[0] is the first)
};
long long layout_hash(const dsem_ctx *c) {
  unsigned long long h = 1469598103934665603ULL;
  auto mix = [&](long long v) {
    h ^= (unsigned long long)v;
    h *= 1099511628211ULL;
  };
  for (const auto &g : c->groups) {
    mix(g.G);
    mix(g.nel);
    mix(g.diag);
  }
  mix(c->nmort);
  return (long long)h;
}
long long evb_doubles(const dsem_ctx *c) {
  long long n = 0;
  for (const auto &g : c->groups) n += 15LL * g.nel * g.G * g.G * g.G;
  return n;
}
long long state_bytes(const dsem_ctx *c) {
  return (long long)sizeof(StateHeader) + (long long)sizeof(double) * (c->ncase - 1) +
         (long long)sizeof(double) * ((long long)c->nq + evb_doubles(c));
}
}  // namespace

extern "C" {

int dsem_state_size(const dsem_ctx *c, long long *nbytes) {
  if (!c || !nbytes) return DSEM_ERR_INVALID_ARG;
  *nbytes = state_bytes(c);
  return DSEM_OK;
}

int dsem_save_state(dsem_ctx *c, void *buf, long long nbytes) {
  if (!c || !buf) return fail(c, DSEM_ERR_INVALID_ARG, "null argument");
  if (nbytes < state_bytes(c)) return fail(c, DSEM_ERR_INVALID_ARG, "buffer smaller than dsem_state_size");
  StateHeader h{};
  std::memcpy(h.magic, "DSEMSTAT", 8);
  h.version = 1;
  h.ngrid = c->ngrid;
  h.nmort = c->nmort;
  h.ncase = c->ncase;
  h.ngroups = (long long)c->groups.size();
  h.nq = (long long)c->nq;
  h.nevb = evb_doubles(c);
  h.flags = (c->grad_valid ? 1 : 0) | (c->ev_grad_valid ? 2 : 0) | (c->keep_grad ? 4 : 0);
  h.layout = layout_hash(c);
  char *out = (char *)buf;
  std::memcpy(out, &h, sizeof(h) - sizeof(double));
  double *pre = (double *)(out + offsetof(StateHeader, prestep));
  for (int k = 0; k < c->ncase; ++k) pre[k] = c->case_prestep[k];
  double *data = pre + c->ncase;
  CK(cudaMemcpyAsync(data, c->JQ, c->nq * sizeof(double), cudaMemcpyDeviceToHost, c->st));
  data += c->nq;
  for (auto &g : c->groups) {
    const size_t n = 15ULL * g.nel * g.G * g.G * g.G;
    CK(cudaMemcpyAsync(data, g.EVB, n * sizeof(double), cudaMemcpyDeviceToHost, c->st));
    data += n;
  }
  CK(cudaStreamSynchronize(c->st));
  return DSEM_OK;
}

int dsem_load_state(dsem_ctx *c, const void *buf, long long nbytes) {
  if (!c || !buf) return fail(c, DSEM_ERR_INVALID_ARG, "null argument");
  if (nbytes < (long long)sizeof(StateHeader)) return fail(c, DSEM_ERR_INVALID_ARG, "snapshot too short");
  StateHeader h{};
  std::memcpy(&h, buf, sizeof(h) - sizeof(double));
  if (std::memcmp(h.magic, "DSEMSTAT", 8) != 0 || h.version != 1)
    return fail(c, DSEM_ERR_INVALID_ARG, "not a dsem state snapshot (version 1)");
  if (h.ngrid != c->ngrid || h.nmort != c->nmort || h.ncase != c->ncase || h.nq != (long long)c->nq ||
      h.ngroups != (long long)c->groups.size() || h.nevb != evb_doubles(c) || h.layout != layout_hash(c))
    return fail(c, DSEM_ERR_INVALID_ARG, "snapshot was taken on a different mesh");
  if (nbytes < state_bytes(c)) return fail(c, DSEM_ERR_INVALID_ARG, "snapshot truncated");
  const char *in = (const char *)buf;
  const double *pre = (const double *)(in + offsetof(StateHeader, prestep));
  for (int k = 0; k < c->ncase; ++k) c->case_prestep[k] = pre[k];
  const double *data = pre + c->ncase;
  CK(cudaMemcpyAsync(c->JQ, data, c->nq * sizeof(double), cudaMemcpyHostToDevice, c->st));
  data += c->nq;
  for (auto &g : c->groups) {
    const size_t n = 15ULL * g.nel * g.G * g.G * g.G;
    CK(cudaMemcpyAsync(g.EVB, data, n * sizeof(double), cudaMemcpyHostToDevice, c->st));
    data += n;
  }
  c->grad_valid = (h.flags & 1) != 0;
  c->ev_grad_valid = (h.flags & 2) != 0;
  c->keep_grad = (h.flags & 4) ? 1 : 0;
  long long l = 0;
  int r = enqueue_traces(c, &l);
  if (r) return r;
  CK(cudaStreamSynchronize(c->st));
  return DSEM_OK;
}

int dsem_profile_rhs(dsem_ctx *c, int reps, double *ms) {
  if (!c || !ms || reps <= 0) return fail(c, DSEM_ERR_INVALID_ARG, "bad argument");
  if (c->ncut) return fail(c, DSEM_ERR_INVALID_ARG, "a shard advances with dsem_shard_stage");
  long long l = 0;
  int r;
  if (!c->traces_valid && (r = enqueue_traces(c, &l))) return r;
  cudaEvent_t ev[5];
  for (auto &e : ev) CK(cudaEventCreate(&e));
  double acc[4] = {0, 0, 0, 0};
  const int mode = vol_mode(c, false);
  for (int it = 0; it < reps; ++it) {
    CK(cudaEventRecord(ev[0], c->st));
    for (auto &ml : c->mlists)
      CK(with_G(ml.G, [&](auto g) {
        return Launch<decltype(g)::value>::face_inv(ml.mc, ml.n, c->QF, c->FF, ml.nh, ml.nrm, c->P.gamma, c->st);
      }));
    for (auto &bl : c->blists)
      CK(with_G(bl.G, [&](auto g) {
        return Launch<decltype(g)::value>::face_bnd_inv(bl.mb, bl.n, c->QF, c->FF, bl.nh, bl.nrm, bl.qext,
                                                        bnd_phys(c), c->st);
      }));
    CK(cudaEventRecord(ev[1], c->st));
    for (auto &g : c->groups) {
      VolArgs a{};
      a.JQ = c->JQ + g.q0;
      a.sq = 5LL * g.G * g.G * g.G;
      a.jac = g.jac;
      a.gg = g.gg;
      a.gm = g.gm;
      a.muhg = g.muhg;
      a.QF = c->QF + g.f0;
      a.VF = c->VF + g.f0;
      a.QTI = c->QTI + g.q0;
      a.EVB = g.EVB;
      a.P = c->P;
      CK(with_G(g.G, [&](auto gg) {
        return Launch<decltype(gg)::value>::vol(a, g.nel, g.diag, mode, c->st, c->vol_variant[g.G]);
      }));
    }
    CK(cudaEventRecord(ev[2], c->st));
    for (auto &ml : c->mlists)  // (the update kernel averages the viscous fluxes on fuse_vis contexts)
      if (!c->fuse_vis)
        CK(with_G(ml.G, [&](auto g) { return Launch<decltype(g)::value>::face_vis(ml.mc, ml.n, c->VF, ml.nrm, c->st); }));
    for (auto &bl : c->blists)
      CK(with_G(bl.G, [&](auto g) {
        return Launch<decltype(g)::value>::face_bnd_vis(bl.mb, bl.n, c->VF, bl.nrm, bl.fvext, c->st);
      }));
    CK(cudaEventRecord(ev[3], c->st));
    for (auto &g : c->groups) {
      UpdArgs u{};
      u.JQ = c->JQ + g.q0;
      u.gQ = c->gQ + g.q0;
      u.sq = 5LL * g.G * g.G * g.G;
      u.jac = g.jac;
      u.QTI = c->QTI + g.q0;
      u.FF = c->FF + g.f0;
      u.VF = c->VF + g.f0;
      u.QF = c->QF + g.f0;
      u.flag = c->flag;
      u.re = c->P.re;
      u.r_re = c->P.r_re;
      u.update = 0;
      if (c->fuse_vis) fuse_vis_args(c, g, u);
      CK(with_G(g.G, [&](auto gg) { return Launch<decltype(gg)::value>::update(u, g.nel, c->st); }));
    }
    CK(cudaEventRecord(ev[4], c->st));
    CK(cudaEventSynchronize(ev[4]));
    for (int k = 0; k < 4; ++k) {
      float t = 0.f;
      CK(cudaEventElapsedTime(&t, ev[k], ev[k + 1]));
      acc[k] += t;
    }
  }
  for (auto &e : ev) cudaEventDestroy(e);
  for (int k = 0; k < 4; ++k) ms[k] = acc[k] / reps;
  return DSEM_OK;
}

int dsem_last_timing(const dsem_ctx *c, double *ms, long long *launches) {
  if (!c) return DSEM_ERR_INVALID_ARG;
  if (ms) *ms = c->last_ms;
  if (launches) *launches = c->last_launches;
  return DSEM_OK;
}

}  // extern "C"

// ------------------------------------------------- hooks for the adjoint unit
namespace dsem_int {
int fail(dsem_ctx *c, int code, const std::string &msg) { return ::fail(c, code, msg); }
int stage(dsem_ctx *c, int kk, bool save) {
  long long l = 0;
  return enqueue_stage(c, kk, save, nullptr, &l, true);
}
int traces(dsem_ctx *c) {
  long long l = 0;
  return enqueue_traces(c, &l);
}
int ev(dsem_ctx *c, const double *jq) {
  long long l = 0;
  return enqueue_ev(c, &l, jq);
}
int les(dsem_ctx *c, const double *jq) {
  long long l = 0;
  return enqueue_les(c, &l, jq);
}
// One RK stage of a single-group context with periodic conforming mortars only,
// out of place: state io.jq_in and its raw face traces io.qf_in (both left
// unchanged) -> the updated state io.jq_out and its raw traces io.qf_out.  The
// same kernels and arithmetic as stage(); c->QF receives the averaged traces.
int stage_io(dsem_ctx *c, int kk, bool save, const StageIO &io) {
  if (c->groups.size() != 1 || c->mlists.size() != 1 || c->nnc > 0 || c->ncut > 0 || !c->blists.empty() || kk < 1)
    return fail(c, DSEM_ERR_UNSUPPORTED, "stage_io: one order group and periodic conforming mortars only");
  const Group &g = c->groups[0];
  const MList &ml = c->mlists[0];
  VolArgs a = vol_args(c, g);
  a.JQ = io.jq_in;
  if (io.evb) a.EVB = io.evb;
  UpdArgs u = upd_args(c, g, kk, nullptr);
  u.JQ = io.jq_in;
  u.JQo = io.jq_out;
  u.QF = io.qf_out;
  if (c->fuse_vis) fuse_vis_args(c, g, u);  // the update kernel averages the viscous face fluxes
  const int mode = vol_mode(c, save);
  CK(with_G(g.G, [&](auto gg) -> cudaError_t {
    using Lg = Launch<decltype(gg)::value>;
    cudaError_t e = Lg::face_inv_from(ml.mc, ml.n, io.qf_in, c->QF, c->FF, ml.nh, ml.nrm, c->P.gamma, c->st);
    if (e == cudaSuccess) e = Lg::vol(a, g.nel, g.diag, mode, c->st, c->vol_variant[g.G]);
    if (e == cudaSuccess && !c->fuse_vis) e = Lg::face_vis(ml.mc, ml.n, c->VF, ml.nrm, c->st);
    if (e == cudaSuccess) e = Lg::update(u, g.nel, c->st);
    return e;
  }));
  return DSEM_OK;
}
int set_dt(dsem_ctx *c, const double *dt) { return ::set_dt(c, dt); }
// kept Lobatto arrays of caller element e: [3][5][L*G^2] at host + 15*L*G^2*e' (e' = running
// offset over the caller's elements, returned by lob_offsets)
std::vector<long long> lob_offsets(const dsem_ctx *c) {
  std::vector<long long> off(c->ngrid + 1, 0);
  for (int e = 0; e < c->ngrid; ++e) {
    const int G = c->groups[c->ext_group[e]].G;
    off[e + 1] = off[e] + 15LL * (G + 1) * G * G;
  }
  return off;
}
int lob_download(dsem_ctx *c, double *host) {
  if (!c->QLB || !c->lob_valid) return fail(c, DSEM_ERR_INVALID_ARG, "no kept Lobatto arrays (dsem_keep_lobatto, then step)");
  const auto off = lob_offsets(c);
  for (int e = 0; e < c->ngrid; ++e) {
    const Group &g = c->groups[c->ext_group[e]];
    const long long n = 15LL * (g.G + 1) * g.G * g.G;
    CK(cudaMemcpyAsync(host + off[e], c->QLB + g.l0 + (long long)c->ext_k[e] * n, n * sizeof(double),
                       cudaMemcpyDeviceToHost, c->st));
  }
  CK(cudaStreamSynchronize(c->st));
  return DSEM_OK;
}
// Lobatto arrays of every caller element (lob_offsets layout) to the device, and the saved
// gradients rebuilt from them: the next step's entropy viscosity / Smagorinsky model use them
int lob_upload_grad(dsem_ctx *c, const double *host) {
  if (!c->QLB) {
    int r = dsem_keep_lobatto(c, 1);
    if (r) return r;
    c->keep_lob = false;
  }
  const auto off = lob_offsets(c);
  for (int e = 0; e < c->ngrid; ++e) {
    const Group &g = c->groups[c->ext_group[e]];
    const long long n = 15LL * (g.G + 1) * g.G * g.G;
    CK(cudaMemcpyAsync(c->QLB + g.l0 + (long long)c->ext_k[e] * n, host + off[e], n * sizeof(double),
                       cudaMemcpyHostToDevice, c->st));
  }
  for (auto &g : c->groups) {
    LobArgs a{};
    a.gg = g.gg;
    a.QLB = c->QLB + g.l0;
    a.EVB = g.EVB;
    a.gamma = c->P.gamma;
    CK(with_G(g.G, [&](auto gg) { return Launch<decltype(gg)::value>::lob_grad(a, g.nel, g.diag, c->st); }));
  }
  CK(cudaStreamSynchronize(c->st));
  c->grad_valid = true;
  c->ev_grad_valid = true;
  c->lob_valid = true;
  return DSEM_OK;
}
// the saved gradients are not valid (a restart file whose Lobatto arrays were never computed)
void grad_invalidate(dsem_ctx *c) {
  c->grad_valid = false;
  c->ev_grad_valid = false;
  c->lob_valid = false;
}
int unpack_state(dsem_ctx *c, const double *dev, double *host, int ldx) {
  return unpack_to_host(c, dev, host, ldx, 5, state_offs(c));
}
int check_flag(dsem_ctx *c) { return ::check_flag(c); }
// per-element enstrophy partials of the last stage's gradients with the state
// jq (null: c->JQ) into part (device, [ngrid][5] in internal order); no sync
int eps_enqueue(dsem_ctx *c, const double *jq, double *part, const double *evb) {
  if (!jq) jq = c->JQ;
  if (evb && c->groups.size() != 1) return fail(c, DSEM_ERR_UNSUPPORTED, "eps_enqueue: one order group");
  for (auto &g : c->groups) {
    k_diag<<<g.nel, 128, sizeof(double) * 5 * g.G * g.G * g.G, c->st>>>(jq + g.q0, g.jac, evb ? evb : g.EVB, g.kew,
                                                                         g.G, g.nel, 1, part + g.e0 * 5);
    CK(cudaGetLastError());
  }
  return DSEM_OK;
}
// the two enstrophy sums from host partials, in the caller's element order
void eps_reduce(const dsem_ctx *c, const double *part, double *s, double *s2) {
  double a = 0.0, b = 0.0;
  for (int e = 0; e < c->ngrid; ++e) {
    const auto &g = c->groups[c->ext_group[e]];
    const double *pp = &part[(size_t)(g.e0 + c->ext_k[e]) * 5];
    a += pp[3];
    b += pp[4];
  }
  *s = a;
  *s2 = b;
}
// enstrophy sums of the last stage's gradients, in the caller's element order
int eps_sums(dsem_ctx *c, double *s, double *s2, const double *jq) {
  int r = eps_enqueue(c, jq, c->part);
  if (r) return r;
  c->host_part.resize((size_t)c->ngrid * 5);
  CK(cudaMemcpyAsync(c->host_part.data(), c->part, c->host_part.size() * sizeof(double), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  eps_reduce(c, c->host_part.data(), s, s2);
  return DSEM_OK;
}
}  // namespace dsem_int
