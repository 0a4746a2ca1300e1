// dsem_adjoint.cu -- dsem_adjoint: discrete adjoint of nsteps Runge-Kutta
// steps for J = sum over the last `window` steps of eps_n * dt, eps_n being the
// enstrophy dissipation dsem_diag reports after step n.  No DSEM counterpart.
//
// Forward sweep: the steps as dsem_step runs them; stage states are kept in
// HBM (every stage of every step when snapshots == 0, else binomial
// checkpoints of step states with the steps recomputed in the reverse sweep;
// with entropy viscosity a checkpoint also keeps the gradients its step's
// viscosity reads).
// Reverse sweep, step n = N..1, stage k = kord..1 (2N-storage RK,
// tstep.f90:66-114):  lg += crk_k dt lQ;  lQ += R'(Q_{k-1})^T lg;  lg *= ark_k,
// with the enstrophy terms of eps_n added at stage kord of each window step.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <string>
#include <utility>
#include <vector>

#include "../../include/dsem_gpu.h"
#include "dsem_adjoint.cuh"
#include "dsem_ctx.h"
#include "dsem_host_math.h"

using namespace dsem;

namespace {

#define CKA(call)                                                                                    \
  do {                                                                                               \
    cudaError_t e_ = (call);                                                                         \
    if (e_ != cudaSuccess) return dsem_int::fail(c, DSEM_ERR_CUDA, std::string(#call ": ") + cudaGetErrorString(e_)); \
  } while (0)

int upload_ops_here(dsem_ctx *c) {  // this translation unit's copy of the operator table
  std::vector<double> table(OPS_TOTAL, 0.0);
  for (int G = GMIN; G <= GMAX; ++G) hostmath::operators(G, &table[ops_off(G)], &table[ops_off(G) + G * (G + 1)]);
  CKA(cudaMemcpyToSymbol(c_ops, table.data(), sizeof(double) * OPS_TOTAL));
  return DSEM_OK;
}

struct AdjBuf {
  double *lq = nullptr, *lg = nullptr, *ljq = nullptr;
  double *qfr = nullptr, *lff = nullptr, *lvf = nullptr, *lqf = nullptr, *lqr = nullptr;
  double *lrp = nullptr, *lr = nullptr;
  double *q0 = nullptr;
  std::vector<double *> slots;  // checkpoint slots (step states)
  double *stages = nullptr;     // stage states: all steps (snapshots == 0) or one step
  double *traces = nullptr;     // raw face traces of every stage state (snapshots == 0, when memory allows)
  // entropy viscosity: dJ/dmu of the step being reversed, dJ/d(gradients saved by
  // the previous step's last stage), and those gradients as they were on entry
  double *lmuhg = nullptr, *levb = nullptr, *evb0 = nullptr;
  double *eps_part = nullptr;  // [window][elements][5] enstrophy partials of the window's steps
  double *evbw = nullptr;      // [window][elements][15][G^3] gradients saved by the window steps' last stages
  // entropy viscosity with checkpoints: each slot also keeps the gradients its step's
  // viscosity reads (saved by the step before it) and whether they existed; evb_prev
  // holds those of the step being reversed
  std::vector<double *> slot_evb;
  std::vector<char> slot_valid;
  double *evb_prev = nullptr;
  double *lrb = nullptr;  // boundary faces: per boundary point, dJ/d(1/Re) of the external viscous flux
  double *volscr = nullptr;  // p = 7, 8: the volume adjoint's per element scratch (VolAdjCfg::SCR)
  ~AdjBuf() {
    for (double *p : {lq, lg, ljq, qfr, lff, lvf, lqf, lqr, lrp, lr, q0, stages, traces, lmuhg, levb, evb0,
                      eps_part, evbw, evb_prev, lrb, volscr})
      cudaFree(p);
    for (double *p : slots) cudaFree(p);
    for (double *p : slot_evb) cudaFree(p);
  }
};

// Where a group's slices of the adjoint's buffers start (doubles, or elements for e0)
struct GOff {
  long long q0 = 0, f0 = 0, e0 = 0;  // state, face slots, elements (as the context's)
  long long gq = 0;                  // Gauss points: q0 / 5 (lmuhg)
  long long ev = 0;                  // saved-gradient slots: 3 q0 (levb, evb copies)
  long long scr = 0;                 // the volume adjoint's scratch (VolAdjCfg::SCR per element)
};

struct Adj {
  dsem_ctx *c;
  std::vector<GOff> off;      // per order group
  std::vector<long long> boff;  // per boundary list: first point in b.lrb
  bool single = true;         // one order group, no p-nonconforming mortars: the fused and out-of-place paths
  const BList *bl = nullptr;  // boundary faces (single group): the list, or null
  AdjBuf b;
  double dt = 0.0, s2 = 0.0;
  int nsteps = 0, window = 0;
  long long launches = 0;
  bool ev = false;            // entropy viscosity on
  bool les = false;           // static Smagorinsky on (never together with ev)
  bool visc = false;          // ev or les: a viscosity from the previous step's saved gradients
  bool ev_valid0 = false;     // the gradients behind the first step's viscosity were valid on entry
  bool levb_pending = false;  // b.levb holds the demand on the next-to-reverse step's saved gradients
  bool ckpt = false;          // checkpoints (snapshots > 0): revolve or segments
  int seg_k = 0;              // segments: steps per segment (0: revolve or store-all)
  bool prev_valid = false;    // checkpoints: b.evb_prev holds valid gradients
  bool in_window(int n) const { return n >= nsteps - window; }  // step n (0-based) ends inside the window
  double eps_w() const { return dt * 100.0 * c->P.r_re / s2; }
};

BndPhys bnd_phys(const dsem_ctx *c) {  // as the forward's face launches
  BndPhys P;
  P.gamma = c->P.gamma;
  P.twall = c->twall;
  P.cv = c->P.mach * c->P.mach * c->P.gamma * (c->P.gamma - 1.0);
  P.r_cv = 1.0 / P.cv;
  return P;
}

// f(gc, group, its offsets) for every order group (gc: the order as a type)
template <class F> int each_group(Adj &A, F &&f) {
  for (size_t j = 0; j < A.c->groups.size(); ++j) {
    int r = DSEM_OK;
    const cudaError_t e = with_G(A.c->groups[j].G, [&](auto gc) -> cudaError_t {
      r = f(gc, A.c->groups[j], A.off[j]);
      return cudaSuccess;
    });
    if (e != cudaSuccess) return dsem_int::fail(A.c, DSEM_ERR_UNSUPPORTED, "adjoint: element order not supported");
    if (r) return r;
  }
  return DSEM_OK;
}
template <class L, class F> int each_list(Adj &A, const std::vector<L> &lists, F &&f) {
  for (size_t j = 0; j < lists.size(); ++j) {
    const cudaError_t e = with_G(lists[j].G, [&](auto gc) -> cudaError_t { return f(gc, lists[j], j); });
    if (e != cudaSuccess) return dsem_int::fail(A.c, DSEM_ERR_CUDA, "adjoint: face launch failed");
  }
  return DSEM_OK;
}

// Stands for "each group's own EVB" where a function takes saved gradients (evb)
const double g_evb_groups = 0.0;
#define EVB_GROUPS (&g_evb_groups)
// a group's slice of saved gradients: its own EVB, a slice of a buffer laid out like b.levb, or null
const double *evb_of(const double *evb, const Group &g, const GOff &o) {
  if (evb == EVB_GROUPS) return g.EVB;
  return evb ? evb + o.ev : nullptr;
}

// Boundary faces: their Dirichlet states (and fluxes, into c->FF) from the raw
// traces now in c->QF's boundary slots, as the forward's k_face_bnd_inv.
int bnd_states(Adj &A) {
  dsem_ctx *c = A.c;
  const BndPhys BP = bnd_phys(c);
  A.launches += (long long)c->blists.size();
  return each_list(A, c->blists, [&](auto gc, const BList &bl, size_t) -> cudaError_t {
    return Launch<decltype(gc)::value>::face_bnd_inv(bl.mb, bl.n, c->QF, c->FF, bl.nh, bl.nrm, bl.qext, BP, c->st);
  });
}

// The forward face inputs of the volume kernels into c->QF: with raw = null the stage
// state Qs's raw traces (a copy kept in b.qfr when keep_raw), else a copy of raw; then the
// averaged states of every interior mortar (conforming and p-nonconforming) and the
// boundary faces' Dirichlet states (fluxes into c->FF).
int face_states(Adj &A, const double *Qs, const double *raw, bool keep_raw) {
  dsem_ctx *c = A.c;
  int r;
  if (!raw) {
    r = each_group(A, [&](auto gc, const Group &g, const GOff &o) -> int {
      constexpr int G = decltype(gc)::value;
      TraceArgs ta{};
      ta.JQ = Qs + o.q0;
      ta.sq = 5LL * G * G * G;
      ta.jac = g.jac;
      ta.QF = c->QF + o.f0;
      CKA(Launch<G>::trace(ta, g.nel, c->st));
      ++A.launches;
      return DSEM_OK;
    });
    if (r) return r;
    if (keep_raw) CKA(cudaMemcpyAsync(A.b.qfr, c->QF, c->nface * sizeof(double), cudaMemcpyDeviceToDevice, c->st));
  } else {
    CKA(cudaMemcpyAsync(c->QF, raw, c->nface * sizeof(double), cudaMemcpyDeviceToDevice, c->st));
  }
  r = each_list(A, c->mlists, [&](auto gc, const MList &ml, size_t) -> cudaError_t {
    return Launch<decltype(gc)::value>::face_inv(ml.mc, ml.n, c->QF, c->FF, ml.nh, ml.nrm, c->P.gamma, c->st);
  });
  if (r) return r;
  A.launches += (long long)c->mlists.size();
  if (c->nnc > 0) {
    k_face_nc_inv<<<c->nnc, 128, 0, c->st>>>(c->nc, c->QF, c->FF, c->nc_nh, c->nc_nrm, c->nc_mats, c->P.gamma);
    CKA(cudaGetLastError());
    ++A.launches;
  }
  return bnd_states(A);
}

// The context's flag for "the saved gradients exist" that the step's viscosity model reads
bool &grad_flag(Adj &A) { return A.les ? A.c->grad_valid : A.c->ev_grad_valid; }

// Adjoint of one stage, the RK steps around it fused in: dJ/dQt += cdt dJ/dQ
// before, dJ/dQ += R'^T dJ/dQt and dJ/dQt *= ark after.  eps_w != 0: the stage
// whose gradients enter the enstrophy sum (with the end state's JQ values JQe).
// qraw: the raw face traces of Qs kept by the forward sweep, or null to recompute them.
// The first part (dJ/dQt += cdt dJ/dQ and the face terms) runs here only when
// upd; otherwise the previous stage of the reverse sweep ran it.  With next,
// this stage's last kernel also runs that first part of the stage reversed
// next, with its coefficient cdt_next.  Per order group: the RK parts, the
// volume adjoint and the trace adjoint; per face list: the face adjoints.
int stage_adjoint(Adj &A, const double *Qs, const double *JQe, double eps_w, double cdt, double ark,
                  const double *qraw, const double *levb, bool upd, bool next, double cdt_next) {
  dsem_ctx *c = A.c;
  // forward prerequisites: raw traces (qfr), averaged and boundary states (c->QF).  One
  // group with kept traces: the viscous-face adjoint writes the averages as it goes.
  const bool fused = qraw && A.single;
  const double *qfr = qraw;
  int r;
  if (!fused) {
    if ((r = face_states(A, Qs, qraw, !qraw))) return r;
    if (!qraw) qfr = A.b.qfr;
  } else if (A.bl) {  // the boundary slots' raw traces, turned into their states below
    CKA(cudaMemcpyAsync(c->QF, qraw, c->nface * sizeof(double), cudaMemcpyDeviceToDevice, c->st));
  }
  int nsm = 0;  // one volume block per SM (shared memory): prefetch one wave ahead
  CKA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->dev));
  if (upd) {
    r = each_group(A, [&](auto gc, const Group &g, const GOff &o) -> int {
      constexpr int G = decltype(gc)::value;
      k_upd_adj<G><<<g.nel, 256, 0, c->st>>>(A.b.lg + o.q0, A.b.lq + o.q0, cdt, A.b.lff + o.f0);
      CKA(cudaGetLastError());
      ++A.launches;
      return DSEM_OK;
    });
    if (r) return r;
  }
  r = each_list(A, c->mlists, [&](auto gc, const MList &ml, size_t) -> cudaError_t {
    constexpr int G = decltype(gc)::value;
    const unsigned nb = (unsigned)(((long long)ml.n * G * G + 127) / 128);
    k_face_vis_adj<G><<<nb, 128, 0, c->st>>>(ml.mc, ml.n, A.b.lff, c->P.re, A.b.lvf, ml.nrm, fused ? qraw : nullptr,
                                             c->QF);
    return cudaGetLastError();
  });
  if (r) return r;
  A.launches += (long long)c->mlists.size();
  if (c->nnc > 0) {
    k_face_nc_vis_adj<<<c->nnc, 128, 0, c->st>>>(c->nc, A.b.lff, c->P.re, A.b.lvf, c->nc_nrm, c->nc_mats);
    CKA(cudaGetLastError());
    ++A.launches;
  }
  if (c->nbnd > 0) {
    if (fused && (r = bnd_states(A))) return r;
    r = each_list(A, c->blists, [&](auto gc, const BList &bl, size_t j) -> cudaError_t {
      constexpr int G = decltype(gc)::value;
      const unsigned nbb = (unsigned)(((long long)bl.n * G * G + 127) / 128);
      k_face_bnd_vis_adj<G><<<nbb, 128, 0, c->st>>>(bl.mb, bl.n, A.b.lff, c->P.re, A.b.lvf, bl.nrm, bl.fvext,
                                                    A.b.lrb + A.boff[j]);
      return cudaGetLastError();
    });
    if (r) return r;
    A.launches += (long long)c->blists.size();
  }
  r = each_group(A, [&](auto gc, const Group &g, const GOff &o) -> int {
    constexpr int G = decltype(gc)::value;
    using C = VolAdjCfg<G>;
    static std::atomic<unsigned long long> attr{0}, attr_ev{0};
    CKA(set_smem_once(k_vol_adj<G, false>, C::SMEM, attr));
    if (A.visc) CKA(set_smem_once(k_vol_adj<G, true>, C::SMEM, attr_ev));
    VolAdjArgs va{};
    va.JQ = Qs + o.q0;
    va.jac = g.jac;
    va.gg = g.gg;
    va.gm = g.gm;
    va.QF = c->QF + o.f0;
    va.LQT = A.b.lg + o.q0;
    va.LVF = A.b.lvf + o.f0;
    va.LJQ = A.b.ljq + o.q0;
    va.LQF = A.b.lqf + o.f0;
    va.lr = A.b.lrp + o.e0;
    va.eps_w = eps_w;
    va.JQe = JQe ? JQe + o.q0 : nullptr;
    va.P = c->P;
    if (A.visc) {
      va.muhg = A.les ? g.nuhg : g.muhg;
      va.lmuhg = A.b.lmuhg + o.gq;
      va.levb = levb ? levb + o.ev : nullptr;
      va.les = A.les ? 1 : 0;
    }
    va.scr = A.b.volscr ? A.b.volscr + o.scr : nullptr;
    va.pf = nsm;
    if (A.visc)
      k_vol_adj<G, true><<<g.nel, C::NT, C::SMEM, c->st>>>(va);
    else
      k_vol_adj<G, false><<<g.nel, C::NT, C::SMEM, c->st>>>(va);
    CKA(cudaGetLastError());
    ++A.launches;
    return DSEM_OK;
  });
  if (r) return r;
  r = each_list(A, c->mlists, [&](auto gc, const MList &ml, size_t) -> cudaError_t {
    constexpr int G = decltype(gc)::value;
    const unsigned nb = (unsigned)(((long long)ml.n * G * G + 127) / 128);
    k_face_inv_adj<G><<<nb, 128, 0, c->st>>>(ml.mc, ml.n, qfr, A.b.lff, A.b.lqf, A.b.lqr, ml.nh, ml.nrm, c->P.gamma);
    return cudaGetLastError();
  });
  if (r) return r;
  A.launches += (long long)c->mlists.size();
  if (c->nnc > 0) {
    k_face_nc_inv_adj<<<c->nnc, 128, 0, c->st>>>(c->nc, qfr, A.b.lff, A.b.lqf, A.b.lqr, c->nc_nh, c->nc_nrm,
                                                 c->nc_mats, c->P.gamma);
    CKA(cudaGetLastError());
    ++A.launches;
  }
  if (c->nbnd > 0) {
    const BndPhys BP = bnd_phys(c);
    r = each_list(A, c->blists, [&](auto gc, const BList &bl, size_t) -> cudaError_t {
      constexpr int G = decltype(gc)::value;
      const unsigned nbb = (unsigned)(((long long)bl.n * G * G + 127) / 128);
      k_face_bnd_inv_adj<G><<<nbb, 128, 0, c->st>>>(bl.mb, bl.n, qfr, A.b.lff, A.b.lqf, A.b.lqr, bl.nh, bl.nrm,
                                                    bl.qext, BP);
      return cudaGetLastError();
    });
    if (r) return r;
    A.launches += (long long)c->blists.size();
  }
  return each_group(A, [&](auto gc, const Group &g, const GOff &o) -> int {
    constexpr int G = decltype(gc)::value;
    if (next)
      k_trace_adj<G, true><<<g.nel, 256, 0, c->st>>>(A.b.lqr + o.f0, g.jac, A.b.ljq + o.q0, A.b.lq + o.q0,
                                                      A.b.lg + o.q0, ark, cdt_next, A.b.lff + o.f0);
    else
      k_trace_adj<G, false><<<g.nel, 256, 0, c->st>>>(A.b.lqr + o.f0, g.jac, A.b.ljq + o.q0, A.b.lq + o.q0,
                                                       A.b.lg + o.q0, ark, 0.0, nullptr);
    CKA(cudaGetLastError());
    ++A.launches;
    return DSEM_OK;
  });
}

// The gradients a forward step's last stage saves (into the groups' EVB),
// recomputed by the forward volume kernels themselves (mode VOL_SAVE or VOL_EV_SAVE)
// from that stage's input state Qs and its raw face traces qraw (null: recomputed).
int saved_grads(Adj &A, const double *Qs, const double *qraw, int mode) {
  dsem_ctx *c = A.c;
  int r;
  if (qraw && A.single) {  // the averages from the kept traces
    if (A.bl) CKA(cudaMemcpyAsync(c->QF, qraw, c->nface * sizeof(double), cudaMemcpyDeviceToDevice, c->st));
    r = each_list(A, c->mlists, [&](auto gc, const MList &ml, size_t) -> cudaError_t {
      constexpr int G = decltype(gc)::value;
      const unsigned nbm = (unsigned)(((long long)ml.n * G * G + 127) / 128);
      k_face_avg<G><<<nbm, 128, 0, c->st>>>(ml.mc, ml.n, qraw, c->QF);
      return cudaGetLastError();
    });
    if (r) return r;
    A.launches += (long long)c->mlists.size();
    if ((r = bnd_states(A))) return r;
  } else if ((r = face_states(A, Qs, qraw, false))) {
    return r;
  }
  return each_group(A, [&](auto gc, const Group &g, const GOff &o) -> int {
    constexpr int G = decltype(gc)::value;
    constexpr int NG = G * G * G;
    VolArgs a{};  // the volume kernel with saved gradients: EVB (its fluxes are not used)
    a.JQ = Qs + o.q0;
    a.sq = 5LL * NG;
    a.jac = g.jac;
    a.gg = g.gg;
    a.gm = g.gm;
    a.muhg = g.muhg;
    a.QF = c->QF + o.f0;
    a.VF = c->VF + o.f0;
    a.QTI = c->QTI + o.q0;
    a.EVB = g.EVB;
    a.P = c->P;
    a.ecase = g.ecase;
    a.rec = c->d_rec;
    CKA(Launch<G>::vol(a, g.nel, true, mode, c->st));
    ++A.launches;
    return DSEM_OK;
  });
}

// Direct part of a window step's enstrophy term into dJ/dQ of its end state
// qend, from the gradients its last stage saved: evb (EVB_GROUPS: the groups'
// own; else a buffer laid out like b.levb), or (null) recomputed from that
// stage's input state Qs and raw traces qraw into the groups' EVB.
int eps_direct(Adj &A, const double *Qs, const double *qraw, const double *qend, const double *evb) {
  dsem_ctx *c = A.c;
  if (!evb) {
    const int r = saved_grads(A, Qs, qraw, VOL_SAVE);
    if (r) return r;
    evb = EVB_GROUPS;
  }
  return each_group(A, [&](auto gc, const Group &g, const GOff &o) -> int {
    constexpr int G = decltype(gc)::value;
    k_eps_dir<G><<<g.nel, 128, 0, c->st>>>(qend + o.q0, g.jac, evb_of(evb, g, o), A.eps_w(), A.b.lq + o.q0);
    CKA(cudaGetLastError());
    ++A.launches;
    return DSEM_OK;
  });
}

// Copies between the groups' EVB and a buffer laid out like b.levb
int evb_copy(Adj &A, double *buf, bool to_buf) {
  dsem_ctx *c = A.c;
  return each_group(A, [&](auto gc, const Group &g, const GOff &o) -> int {
    constexpr int G = decltype(gc)::value;
    const size_t n = (size_t)g.nel * 15 * G * G * G * sizeof(double);
    if (to_buf)
      CKA(cudaMemcpyAsync(buf + o.ev, g.EVB, n, cudaMemcpyDeviceToDevice, c->st));
    else
      CKA(cudaMemcpyAsync(g.EVB, buf + o.ev, n, cudaMemcpyDeviceToDevice, c->st));
    return DSEM_OK;
  });
}

// Entropy viscosity (or Smagorinsky) for the reverse sweep of a step whose start state is Qn:
// first the gradients that fed it, saved by the previous step's last stage
// (when that stage's input state Qprev is kept: recomputed from it and its raw
// face traces; else with checkpoints: copied aside before the step's
// recomputation, keep_prev; else kept from entry for the first step), then
// the viscosity itself (k_ev / k_les, into the groups' muhg / nuhg).  *valid: whether those
// gradients existed.
int ev_forward(Adj &A, const double *Qn, const double *Qprev, const double *qraw_prev, bool *valid) {
  dsem_ctx *c = A.c;
  bool ok = true;
  int r;
  if (Qprev) {
    if ((r = saved_grads(A, Qprev, qraw_prev, A.les ? VOL_SAVE : VOL_EV_SAVE))) return r;
  } else if (A.ckpt) {  // kept before the step's recomputation overwrote them
    ok = A.prev_valid;
    if (ok && (r = evb_copy(A, A.b.evb_prev, false))) return r;
  } else if (A.ev_valid0) {
    if ((r = evb_copy(A, A.b.evb0, false))) return r;
  } else {
    ok = false;
  }
  r = each_group(A, [&](auto gc, const Group &g, const GOff &o) -> int {
    constexpr int G = decltype(gc)::value;
    constexpr int NG = G * G * G;
    if (A.les) {  // simpleSmag (k_les), into the group's nuhg
      LesArgs a{};
      a.JQ = Qn + o.q0;
      a.sq = 5LL * NG;
      a.jac = g.jac;
      a.hd = g.hd;
      a.EVB = g.EVB;
      a.nuhg = g.nuhg;
      a.sens = g.sens;
      a.sensors = 0;
      a.valid = ok ? 1 : 0;
      a.re = c->P.re;
      a.cs = c->les_cs;
      a.numax = c->les_numax;
      a.ecase = g.ecase;
      a.rec = c->d_rec;
      CKA(Launch<G>::les(a, g.nel, c->st));
    } else {
      EvArgs e{};
      e.JQ = Qn + o.q0;
      e.sq = 5LL * NG;
      e.jac = g.jac;
      e.hd = g.hd;
      e.EVB = g.EVB;
      e.muhg = g.muhg;
      e.valid = ok ? 1 : 0;
      e.P = c->P;
      e.ecase = g.ecase;
      e.rec = c->d_rec;
      CKA(Launch<G>::ev(e, g.nel, c->st));
    }
    ++A.launches;
    return DSEM_OK;
  });
  if (r) return r;
  CKA(cudaMemsetAsync(A.b.lmuhg, 0, (size_t)(c->nq / 5) * sizeof(double), c->st));
  *valid = ok;
  return DSEM_OK;
}

// dJ/dmu (or dJ/dnu_t) of the reversed step into dJ/dQn (b.lq) and the previous step's saved
// gradients (b.levb)
int ev_adjoint(Adj &A, const double *Qn) {
  dsem_ctx *c = A.c;
  return each_group(A, [&](auto gc, const Group &g, const GOff &o) -> int {
    constexpr int G = decltype(gc)::value;
    if (A.les) {
      LesAdjArgs e{};
      e.JQ = Qn + o.q0;
      e.jac = g.jac;
      e.hd = g.hd;
      e.EVB = g.EVB;
      e.LNU = A.b.lmuhg + o.gq;
      e.LQ = A.b.lq + o.q0;
      e.LEVB = A.b.levb + o.ev;
      e.LR = A.b.lrp + o.e0;
      e.re = c->P.re;
      e.cs = c->les_cs;
      e.numax = c->les_numax;
      e.valid = 1;
      k_les_adj<G><<<g.nel, 128, 0, c->st>>>(e);
    } else {
      EvAdjArgs e{};
      e.JQ = Qn + o.q0;
      e.jac = g.jac;
      e.hd = g.hd;
      e.EVB = g.EVB;
      e.LMU = A.b.lmuhg + o.gq;
      e.LQ = A.b.lq + o.q0;
      e.LEVB = A.b.levb + o.ev;
      e.P = c->P;
      k_ev_adj<G><<<g.nel, 128, 0, c->st>>>(e);
    }
    CKA(cudaGetLastError());
    ++A.launches;
    return DSEM_OK;
  });
}

// Reverse of step n, its stage input states at st[0..kord) and its end state at
// qend; qf[0..kord): their raw face traces, or null.  With entropy viscosity,
// qprev / qfprev: the previous step's last stage input state and its raw traces
// (null for the first step).  evb: the gradients step n's last stage saved, or
// null to recompute them (used when step n is in the objective's window).
int reverse_step(Adj &A, int n, double *const *st, const double *qend, double *const *qf = nullptr,
                 const double *qprev = nullptr, const double *qfprev = nullptr, const double *evb = nullptr) {
  dsem_ctx *c = A.c;
  const bool win = A.in_window(n);
  if (win) {  // d eps_n / d JQ_n through the JQ values of the enstrophy sum
    int r = eps_direct(A, st[c->kord - 1], qf ? qf[c->kord - 1] : nullptr, qend, evb);
    if (r) return r;
  }
  bool ev_valid = false;
  if (A.visc) {
    const int r = ev_forward(A, st[0], qprev, qfprev, &ev_valid);
    if (r) return r;
  }
  for (int kk = c->kord; kk >= 1; --kk) {
    const bool eps_here = win && kk == c->kord;
    const double *levb = (A.visc && kk == c->kord && A.levb_pending) ? A.b.levb : nullptr;
    int r = stage_adjoint(A, st[kk - 1], qend, eps_here ? A.eps_w() : 0.0, c->crk[kk - 1] * A.dt,
                          c->ark[kk - 1], qf ? qf[kk - 1] : nullptr, levb, kk == c->kord, kk > 1,
                          kk > 1 ? c->crk[kk - 2] * A.dt : 0.0);
    if (r) return r;
  }
  if (A.visc) {  // the step's viscosity, from its start state and the previous step's gradients
    if (ev_valid) {
      const int r = ev_adjoint(A, st[0]);
      if (r) return r;
    }
    A.levb_pending = ev_valid && n > 0;  // gradients saved inside the run (not held fixed from before it)
  }
  return DSEM_OK;
}

// One forward step from c->JQ; stage input states copied to st[0..kord) when st
// != nullptr, their raw face traces (c->QF at the stage start) to qf[0..kord)
// when qf != nullptr.  With st, qf, jq_next and qf_next all given the step runs
// out of place instead: st[0] and qf[0] already hold its start state and raw
// traces, each stage writes the next stage's into st[kk] and qf[kk], and the
// last stage writes the end state and its raw traces into jq_next and qf_next
// (no copies; the same kernels and arithmetic), and the gradients it saves into
// evb_slot when given.
int forward_step(Adj &A, int n, double *const *st, double *eps_part, double *const *qf = nullptr,
                 double *jq_next = nullptr, double *qf_next = nullptr, double *evb_slot = nullptr) {
  dsem_ctx *c = A.c;
  const bool win = A.in_window(n);
  const bool oop = st && qf && jq_next && qf_next;
  for (int kk = 1; kk <= c->kord; ++kk) {
    if (!oop && st) CKA(cudaMemcpyAsync(st[kk - 1], c->JQ, c->nq * sizeof(double), cudaMemcpyDeviceToDevice, c->st));
    if (!oop && qf)
      CKA(cudaMemcpyAsync(qf[kk - 1], c->QF, c->nface * sizeof(double), cudaMemcpyDeviceToDevice, c->st));
    if (A.visc && kk == 1) {  // the step's entropy or Smagorinsky viscosity (tstep.f90:36-43)
      const int r = A.les ? dsem_int::les(c, oop ? st[0] : nullptr) : dsem_int::ev(c, oop ? st[0] : nullptr);
      if (r) return r;
    }
    const bool save = (win || A.visc) && kk == c->kord;
    int r;
    if (oop) {
      const bool last = kk == c->kord;
      const dsem_int::StageIO io{st[kk - 1], qf[kk - 1], last ? jq_next : st[kk], last ? qf_next : qf[kk],
                                 last ? evb_slot : nullptr};
      r = dsem_int::stage_io(c, kk, save, io);
    } else {
      r = dsem_int::stage(c, kk, save);
    }
    if (r) return r;
    A.launches += 2 * (long long)c->groups.size() + 2 * (long long)c->mlists.size();
  }
  if (A.visc) grad_flag(A) = true;  // the last stage saved the gradients of the next viscosity
  if (win && eps_part) {  // the step's enstrophy partials, summed on the host after the sweep
    int r = dsem_int::eps_enqueue(c, oop ? jq_next : nullptr, eps_part, oop ? evb_slot : nullptr);
    if (r) return r;
    ++A.launches;
  }
  return DSEM_OK;
}

// Captures the launches of f() on the context's stream and replays them through
// *gx, which is instantiated on first use and updated in place afterwards (the
// same launches with other pointers and scalars).
template <class F> int replay(dsem_ctx *c, cudaGraphExec_t *gx, F &&f) {
  cudaGraph_t graph = nullptr;
  cudaError_t ec = cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal);
  if (ec != cudaSuccess) return dsem_int::fail(c, DSEM_ERR_CUDA, "adjoint: cudaStreamBeginCapture failed");
  const int r = f();
  ec = cudaStreamEndCapture(c->st, &graph);
  if (r) {
    if (graph) cudaGraphDestroy(graph);
    return r;
  }
  if (ec != cudaSuccess) return dsem_int::fail(c, DSEM_ERR_CUDA, "adjoint: cudaStreamEndCapture failed");
  if (*gx) {
    cudaGraphExecUpdateResultInfo info;
    if (cudaGraphExecUpdate(*gx, graph, &info) != cudaSuccess) {
      cudaGetLastError();
      cudaGraphExecDestroy(*gx);
      *gx = nullptr;
    }
  }
  if (!*gx) ec = cudaGraphInstantiate(gx, graph, 0);
  cudaGraphDestroy(graph);
  if (ec != cudaSuccess) return dsem_int::fail(c, DSEM_ERR_CUDA, "adjoint: cudaGraphInstantiate failed");
  ec = cudaGraphLaunch(*gx, c->st);
  if (ec != cudaSuccess) return dsem_int::fail(c, DSEM_ERR_CUDA, "adjoint: cudaGraphLaunch failed");
  return DSEM_OK;
}

// bytes of all groups' saved gradients (15 G^3 doubles per element: 3 nq)
size_t evb_bytes(const Adj &A) { return (size_t)3 * A.c->nq * sizeof(double); }

// The state of slot si into the context; with entropy viscosity also the
// gradients behind the viscosity of the slot's step and their validity.
int load_slot(Adj &A, int si) {
  dsem_ctx *c = A.c;
  CKA(cudaMemcpyAsync(c->JQ, A.b.slots[si], c->nq * sizeof(double), cudaMemcpyDeviceToDevice, c->st));
  if (A.visc) {
    if (int r = evb_copy(A, A.b.slot_evb[si], false)) return r;
    grad_flag(A) = A.b.slot_valid[si] != 0;
  }
  return dsem_int::traces(c);
}

// The context's state into slot si (and, with entropy viscosity, the gradients the
// next step's viscosity reads).
int save_slot(Adj &A, int si) {
  dsem_ctx *c = A.c;
  CKA(cudaMemcpyAsync(A.b.slots[si], c->JQ, c->nq * sizeof(double), cudaMemcpyDeviceToDevice, c->st));
  if (A.visc) {
    if (int r = evb_copy(A, A.b.slot_evb[si], true)) return r;
    A.b.slot_valid[si] = grad_flag(A) ? 1 : 0;
  }
  return DSEM_OK;
}

// Before the recomputation of a step about to be reversed: the gradients its
// viscosity reads, which that step's last stage overwrites.
int keep_prev(Adj &A) {
  if (!A.visc) return DSEM_OK;
  if (int r = evb_copy(A, A.b.evb_prev, true)) return r;
  A.prev_valid = grad_flag(A);
  return DSEM_OK;
}

// binomial checkpoint count beta(s, t) = C(s + t, s), saturated
long long beta(int s, int t) {
  long double v = 1.0L;
  for (int i = 1; i <= s; ++i) {
    v = v * (t + i) / i;
    if (v > 4e18L) return (long long)4e18;
  }
  return (long long)(v + 0.5L);
}

// Binomial split of l steps with nfree free slots: the length of the left
// segment, the left segment's beta(nfree, t - 1) for the smallest t with
// beta(nfree, t) >= l.
long long split_left(long long l, int nfree) {
  int t = 1;
  while (beta(nfree, t) < l) ++t;
  return std::max<long long>(1, std::min<long long>(l - 1, beta(nfree, t - 1)));
}

// The snapshots revolve takes on its first descent, along the right edge of the
// recursion from revolve(0, nsteps, 0, 1): (step index m, slot) pairs.  The
// first forward sweep saves them as it passes, so the reverse sweep starts with
// revolve_spine and skips re-advancing to them.
std::vector<std::pair<int, int>> spine(int nsteps, int nslots) {
  std::vector<std::pair<int, int>> v;
  int i = 0, sfree = 1;
  while (nsteps - i > 1 && nslots - sfree > 0) {
    const int m = i + (int)split_left(nsteps - i, nslots - sfree);
    v.emplace_back(m, sfree);
    i = m;
    ++sfree;
  }
  return v;
}

// Reverse steps [i, j) whose start state is in slot si; slots [sfree, end) are free.
int revolve(Adj &A, int i, int j, int si, int sfree) {
  dsem_ctx *c = A.c;
  const int nfree = (int)A.b.slots.size() - sfree;
  std::vector<double *> st(c->kord), qf;
  for (int k = 0; k < c->kord; ++k) st[k] = A.b.stages + (size_t)k * c->nq;
  if (A.b.traces)  // the raw face traces of the step about to be reversed
    for (int k = 0; k < c->kord; ++k) qf.push_back(A.b.traces + (size_t)k * c->nface);
  double *const *qfp = qf.empty() ? nullptr : qf.data();
  if (j - i == 1) {
    int r = load_slot(A, si);
    if (r) return r;
    if ((r = keep_prev(A)) || (r = forward_step(A, i, st.data(), nullptr, qfp))) return r;
    return reverse_step(A, i, st.data(), c->JQ, qfp, nullptr, nullptr, EVB_GROUPS);
  }
  if (nfree == 0) {  // no free slot: re-advance from slot si for every step
    for (int m = j - 1; m >= i; --m) {
      int r = load_slot(A, si);
      if (r) return r;
      for (int n = i; n < m; ++n)
        if ((r = forward_step(A, n, nullptr, nullptr))) return r;
      if ((r = keep_prev(A)) || (r = forward_step(A, m, st.data(), nullptr, qfp))) return r;
      if ((r = reverse_step(A, m, st.data(), c->JQ, qfp, nullptr, nullptr, EVB_GROUPS))) return r;
    }
    return DSEM_OK;
  }
  const int m = i + (int)split_left(j - i, nfree);
  int r = load_slot(A, si);
  if (r) return r;
  for (int n = i; n < m; ++n)
    if ((r = forward_step(A, n, nullptr, nullptr))) return r;
  if ((r = save_slot(A, sfree))) return r;
  if ((r = revolve(A, m, j, sfree, sfree + 1))) return r;
  return revolve(A, i, m, si, sfree);
}

// revolve(i, j, si, sfree) with the snapshots of spine() already in their slots
int revolve_spine(Adj &A, int i, int j, int si, int sfree) {
  const int nfree = (int)A.b.slots.size() - sfree;
  if (j - i == 1 || nfree == 0) return revolve(A, i, j, si, sfree);
  const int m = i + (int)split_left(j - i, nfree);
  const int r = revolve_spine(A, m, j, sfree, sfree + 1);  // slot sfree holds the state after m steps
  if (r) return r;
  return revolve(A, i, m, si, sfree);
}

// ---- two-level scheme (DSEM_ADJ_SEGMENTS): b.stages / b.traces hold the stage
// states and raw face traces of one segment, its step i at [i * kord, (i + 1) * kord).

// Steps [b, e) out of place through the segment stash, starting from c->JQ and
// c->QF (copied into the stash's first slot); the segment's end state and its
// raw traces go to c->JQ and c->QF.  eps_part: the window's enstrophy partials
// (the first sweep), or null (a recomputation).  With b.evbw the gradients that
// each window step's last stage saves go to its slot [step in segment].
int seg_forward(Adj &A, int b, int e, double *eps_part, cudaGraphExec_t *gx) {
  dsem_ctx *c = A.c;
  const int kord = c->kord;
  const size_t nq = c->nq, nf = c->nface, npart = (size_t)c->ngrid * 5;
  const size_t nevb = (size_t)3 * c->nq;
  CKA(cudaMemcpyAsync(A.b.stages, c->JQ, nq * sizeof(double), cudaMemcpyDeviceToDevice, c->st));
  CKA(cudaMemcpyAsync(A.b.traces, c->QF, nf * sizeof(double), cudaMemcpyDeviceToDevice, c->st));
  for (int n = b; n < e; ++n) {
    const int i = n - b;
    std::vector<double *> st, qf;
    for (int k = 0; k < kord; ++k) {
      st.push_back(A.b.stages + ((size_t)i * kord + k) * nq);
      qf.push_back(A.b.traces + ((size_t)i * kord + k) * nf);
    }
    const bool last = n + 1 == e, win = A.in_window(n);
    double *jq_next = last ? c->JQ : A.b.stages + (size_t)(i + 1) * kord * nq;
    double *qf_next = last ? c->QF : A.b.traces + (size_t)(i + 1) * kord * nf;
    double *part = (win && eps_part) ? eps_part + (size_t)(n - (A.nsteps - A.window)) * npart : nullptr;
    double *evb = (win && A.b.evbw) ? A.b.evbw + (size_t)i * nevb : nullptr;
    auto f = [&] { return forward_step(A, n, st.data(), part, qf.data(), jq_next, qf_next, evb); };
    const int r = i == 0 ? f() : replay(c, &gx[win ? 1 : 0], f);
    if (r) return r;
  }
  return DSEM_OK;
}

// Reverse of steps [e - 1 .. b] from the segment stash that seg_forward filled
// (the end state in c->JQ).  Each step's viscosity reads gradients recomputed
// from the previous step's stored last stage, except the segment's first step,
// whose gradients keep_prev copied aside.  first: the first segment reversed.
int seg_reverse(Adj &A, int b, int e, bool first, cudaGraphExec_t *gx) {
  dsem_ctx *c = A.c;
  const int kord = c->kord;
  const size_t nq = c->nq, nf = c->nface;
  const size_t nevb = (size_t)3 * c->nq;
  for (int m = e - 1; m >= b; --m) {
    const int i = m - b;
    std::vector<double *> st, qf;
    for (int k = 0; k < kord; ++k) {
      st.push_back(A.b.stages + ((size_t)i * kord + k) * nq);
      qf.push_back(A.b.traces + ((size_t)i * kord + k) * nf);
    }
    const double *qend = m + 1 < e ? A.b.stages + (size_t)(i + 1) * kord * nq : c->JQ;
    const double *qprev = m > b ? A.b.stages + ((size_t)(i - 1) * kord + kord - 1) * nq : nullptr;
    const double *qfprev = m > b ? A.b.traces + ((size_t)(i - 1) * kord + kord - 1) * nf : nullptr;
    const double *evb = A.visc ? EVB_GROUPS : ((A.in_window(m) && A.b.evbw) ? A.b.evbw + (size_t)i * nevb : nullptr);
    auto f = [&] { return reverse_step(A, m, st.data(), qend, qf.data(), qprev, qfprev, evb); };
    const int r = ((first && m == e - 1) || (A.visc && m == b)) ? f() : replay(c, &gx[A.in_window(m) ? 1 : 0], f);
    if (r) return r;
  }
  return DSEM_OK;
}

}  // namespace

extern "C" int dsem_set_adjoint_scheme(dsem_ctx *c, int scheme) {
  if (!c) return dsem_int::fail(c, DSEM_ERR_INVALID_ARG, "null context");
  if (scheme != DSEM_ADJ_REVOLVE && scheme != DSEM_ADJ_SEGMENTS)
    return dsem_int::fail(c, DSEM_ERR_INVALID_ARG, "adjoint scheme: DSEM_ADJ_REVOLVE or DSEM_ADJ_SEGMENTS");
  c->adj_scheme = scheme;
  return DSEM_OK;
}

#ifdef DSEM_PHASE_TIMING
extern "C" int dsem_debug_phase_cycles_adj(unsigned long long *out, int reset) {
  cudaError_t e = cudaMemcpyFromSymbol(out, ::g_phase_cycles, sizeof(unsigned long long) * 32);
  if (reset) {
    unsigned long long z[32] = {};
    cudaMemcpyToSymbol(::g_phase_cycles, z, sizeof(z));
  }
  return (int)e;
}
#endif

extern "C" int dsem_adjoint(dsem_ctx *c, double dt, int nsteps, int window, int snapshots, double *J, double *dJdQ0,
                            int ldx, double *dJdinvRe, double *ms) {
  if (!c) return dsem_int::fail(c, DSEM_ERR_INVALID_ARG, "null context");
  if (nsteps < 1 || window < 0 || window > nsteps || snapshots < 0 || !(dt > 0.0))
    return dsem_int::fail(c, DSEM_ERR_INVALID_ARG, "adjoint: need nsteps >= 1, 0 <= window <= nsteps, snapshots >= 0, dt > 0");
  bool diag = true;
  int gmax = 0;
  for (const Group &g : c->groups) {
    diag = diag && g.diag;
    gmax = std::max(gmax, g.G);
  }
  if (c->ncase != 1 || !diag || (c->les && (c->shock || c->les_sensors)) || c->ncut > 0)
    return dsem_int::fail(c, DSEM_ERR_UNSUPPORTED,
                          "adjoint: one case, axis-aligned elements, no LES together with entropy viscosity or the "
                          "LES sensors, no sharding");
  if (dJdQ0 && ldx < gmax) return dsem_int::fail(c, DSEM_ERR_INVALID_ARG, "ldx smaller than the number of Gauss points");
  int r = upload_ops_here(c);
  if (r) return r;
  Adj A;
  A.c = c;
  A.single = c->groups.size() == 1 && c->nnc == 0;
  A.bl = (A.single && c->nbnd > 0) ? &c->blists[0] : nullptr;
  {  // the groups' slices of the buffers
    long long scr = 0;
    for (const Group &g : c->groups) {
      GOff o;
      o.q0 = g.q0;
      o.f0 = g.f0;
      o.e0 = g.e0;
      o.gq = g.q0 / 5;
      o.ev = 3 * g.q0;
      o.scr = scr;
      with_G(g.G, [&](auto gc) -> cudaError_t {
        scr += (long long)VolAdjCfg<decltype(gc)::value>::SCR * g.nel;
        return cudaSuccess;
      });
      A.off.push_back(o);
    }
    // p = 7, 8: the volume adjoint's arrays that do not fit shared memory
    if (scr && cudaMalloc(&A.b.volscr, (size_t)scr * sizeof(double)) != cudaSuccess) {
      cudaGetLastError();
      return dsem_int::fail(c, DSEM_ERR_NOMEM, "adjoint: not enough device memory for the volume scratch");
    }
  }
  A.dt = dt;
  A.nsteps = nsteps;
  A.window = window;
  const size_t nq = c->nq, nf = c->nface, bq = nq * sizeof(double), bf = nf * sizeof(double);
  const int kord = c->kord;
  for (double **p : {&A.b.lq, &A.b.lg, &A.b.ljq, &A.b.q0}) CKA(cudaMalloc(p, bq));
  for (double **p : {&A.b.qfr, &A.b.lff, &A.b.lvf, &A.b.lqf, &A.b.lqr}) CKA(cudaMalloc(p, bf));
  CKA(cudaMalloc(&A.b.lrp, (size_t)c->ngrid * sizeof(double)));
  size_t nbpt = 0;  // boundary points, per list
  for (const BList &bl : c->blists) {
    A.boff.push_back((long long)nbpt);
    nbpt += (size_t)bl.n * bl.G * bl.G;
  }
  if (nbpt) {
    CKA(cudaMalloc(&A.b.lrb, nbpt * sizeof(double)));
    CKA(cudaMemsetAsync(A.b.lrb, 0, nbpt * sizeof(double), c->st));
  }
  A.ev = c->shock != 0;
  A.les = c->les != 0;
  A.visc = A.ev || A.les;
  if (A.visc) {
    CKA(cudaMalloc(&A.b.lmuhg, (nq / 5) * sizeof(double)));
    CKA(cudaMalloc(&A.b.levb, evb_bytes(A)));
    A.ev_valid0 = grad_flag(A);
    if (A.ev_valid0) {  // the gradients behind the first step's viscosity
      CKA(cudaMalloc(&A.b.evb0, evb_bytes(A)));
      if ((r = evb_copy(A, A.b.evb0, true))) return r;
    }
  }
  CKA(cudaMalloc(&A.b.lr, sizeof(double)));
  // DSEM_ADJOINT_LEAN=1 takes the paths used when device memory is short: no
  // optional trace or gradient slots and no segment stash (the same results,
  // bit for bit, more work)
  const char *lean_env = std::getenv("DSEM_ADJOINT_LEAN");
  const bool lean = lean_env && lean_env[0] == '1';
  // two-level scheme: snapshots at the starts of segments of seg_k steps, and one
  // segment's stage states and raw traces (the stash); revolve when they do not fit
  int seg_k = 0, nseg = 0;
  if (snapshots > 0 && c->adj_scheme == DSEM_ADJ_SEGMENTS && !lean && A.single && c->nbnd == 0) {
    seg_k = (nsteps + snapshots - 1) / snapshots;
    nseg = (nsteps + seg_k - 1) / seg_k;
    if (cudaMalloc(&A.b.stages, (size_t)seg_k * kord * bq) != cudaSuccess ||
        cudaMalloc(&A.b.traces, (size_t)seg_k * kord * bf) != cudaSuccess) {
      cudaGetLastError();
      cudaFree(A.b.stages);
      cudaFree(A.b.traces);
      A.b.stages = A.b.traces = nullptr;
      seg_k = nseg = 0;
    }
  }
  A.seg_k = seg_k;
  if (!seg_k) {
    const size_t nstage = snapshots == 0 ? (size_t)nsteps * kord : (size_t)kord;
    if (cudaMalloc(&A.b.stages, nstage * bq) != cudaSuccess) {
      cudaGetLastError();
      return dsem_int::fail(c, DSEM_ERR_NOMEM, "adjoint: not enough device memory for the stage states (use snapshots > 0)");
    }
    // raw face traces of every kept stage state (with snapshots: of the step being reversed)
    if (lean || cudaMalloc(&A.b.traces, nstage * bf) != cudaSuccess) {
      cudaGetLastError();  // not enough memory: the reverse sweep recomputes the traces
      A.b.traces = nullptr;
    }
  }
  A.ckpt = snapshots > 0;
  const int nslots = seg_k ? nseg : snapshots;
  for (int s = 0; s < nslots; ++s) {
    double *p = nullptr, *pe = nullptr;
    if (cudaMalloc(&p, bq) != cudaSuccess || (A.visc && cudaMalloc(&pe, evb_bytes(A)) != cudaSuccess)) {
      cudaGetLastError();
      cudaFree(p);
      return dsem_int::fail(c, DSEM_ERR_NOMEM, "adjoint: not enough device memory for the snapshots");
    }
    A.b.slots.push_back(p);
    if (A.visc) {
      A.b.slot_evb.push_back(pe);
      A.b.slot_valid.push_back(0);
    }
  }
  if (A.visc && A.ckpt) CKA(cudaMalloc(&A.b.evb_prev, evb_bytes(A)));
  std::vector<double> tmp(1, dt);
  if ((r = dsem_int::set_dt(c, tmp.data()))) return r;
  cudaEvent_t e0, e1;
  CKA(cudaEventCreate(&e0));
  CKA(cudaEventCreate(&e1));
  CKA(cudaEventRecord(e0, c->st));
  CKA(cudaMemcpyAsync(A.b.q0, c->JQ, bq, cudaMemcpyDeviceToDevice, c->st));
  CKA(cudaMemsetAsync(c->flag, 0, sizeof(int), c->st));
  if ((r = dsem_int::traces(c))) return r;
  // with every stage state and its raw traces kept, the sweep runs out of place
  // through the stash: its first slot starts with the initial state and traces
  const bool oop = snapshots == 0 && A.b.traces && A.single && c->nbnd == 0;  // out-of-place stages: one group, periodic faces
  if (oop) {
    CKA(cudaMemcpyAsync(A.b.stages, c->JQ, bq, cudaMemcpyDeviceToDevice, c->st));
    CKA(cudaMemcpyAsync(A.b.traces, c->QF, bf, cudaMemcpyDeviceToDevice, c->st));
  }
  // ---- forward sweep
  std::vector<double> s_win;
  const size_t npart = (size_t)c->ngrid * 5;
  if (window > 0) CKA(cudaMalloc(&A.b.eps_part, (size_t)window * npart * sizeof(double)));
  // the gradients saved by each window step's last stage, for the reverse
  // sweep's direct enstrophy term (else recomputed there)
  const size_t nevb = (size_t)3 * c->nq;
  if (oop && !A.visc && window > 0 && !lean &&
      cudaMalloc(&A.b.evbw, (size_t)window * nevb * sizeof(double)) != cudaSuccess) {
    cudaGetLastError();
    A.b.evbw = nullptr;
  }
  if (seg_k && !A.visc && window > 0 &&  // segments: one slot per step of a segment
      cudaMalloc(&A.b.evbw, (size_t)seg_k * nevb * sizeof(double)) != cudaSuccess) {
    cudaGetLastError();
    A.b.evbw = nullptr;
  }
  {
    // after the first (eager) step, steps are captured and replayed as CUDA
    // graphs, one per kind of step (inside or outside the window); the window's
    // enstrophy partials stay on the device until the sweep ends, so the host
    // never waits for the GPU between steps
    cudaGraphExec_t gx[2] = {nullptr, nullptr};
    auto drop = [&]() {
      for (auto &x : gx)
        if (x) cudaGraphExecDestroy(x);
    };
    std::vector<std::pair<int, int>> sp;
    if (snapshots > 0 && !seg_k) sp = spine(nsteps, snapshots);
    size_t ksp = 0;  // next snapshot of the spine
    for (int n = 0; n < nsteps; ++n) {
      if (ksp < sp.size() && sp[ksp].first == n) {  // the state after n steps, for the reverse sweep
        if ((r = save_slot(A, sp[ksp].second))) return drop(), r;
        ++ksp;
      }
      if (seg_k && n % seg_k == 0) {  // segments: the state at each segment's start
        if (n > 0 && (r = save_slot(A, n / seg_k))) return drop(), r;
        if (n / seg_k == nseg - 1) {  // the last segment runs through the stash, ready to reverse
          if ((r = keep_prev(A)) || (r = seg_forward(A, n, nsteps, A.b.eps_part, gx))) return drop(), r;
          break;
        }
      }
      std::vector<double *> st, qf;
      if (snapshots == 0)
        for (int k = 0; k < kord; ++k) {
          st.push_back(A.b.stages + ((size_t)n * kord + k) * nq);
          if (A.b.traces) qf.push_back(A.b.traces + ((size_t)n * kord + k) * nf);
        }
      double *const *stp = snapshots == 0 ? st.data() : nullptr;
      double *const *qfp = qf.empty() ? nullptr : qf.data();
      double *jq_next = nullptr, *qf_next = nullptr;  // out of place: where the step's end state goes
      if (oop) {
        const bool last = n + 1 == nsteps;
        jq_next = last ? c->JQ : A.b.stages + (size_t)(n + 1) * kord * nq;
        qf_next = last ? c->QF : A.b.traces + (size_t)(n + 1) * kord * nf;
      }
      const bool win = A.in_window(n);
      double *part = win ? A.b.eps_part + (size_t)(n - (nsteps - window)) * npart : nullptr;
      double *evb = (win && A.b.evbw) ? A.b.evbw + (size_t)(n - (nsteps - window)) * nevb : nullptr;
      if (n == 0) {
        if ((r = forward_step(A, n, stp, part, qfp, jq_next, qf_next, evb))) return drop(), r;
        continue;
      }
      if ((r = replay(c, &gx[win ? 1 : 0],
                      [&] { return forward_step(A, n, stp, part, qfp, jq_next, qf_next, evb); })))
        return drop(), r;
    }
    drop();
  }
  if (window > 0) {  // the window's enstrophy sums, step by step in the caller's element order
    std::vector<double> hp((size_t)window * npart);
    CKA(cudaMemcpyAsync(hp.data(), A.b.eps_part, hp.size() * sizeof(double), cudaMemcpyDeviceToHost, c->st));
    CKA(cudaStreamSynchronize(c->st));
    for (int w = 0; w < window; ++w) {
      double sv = 0.0, s2 = 0.0;
      dsem_int::eps_reduce(c, hp.data() + (size_t)w * npart, &sv, &s2);
      s_win.push_back(sv);
      A.s2 = s2;  // the normalisation: the window's last step
    }
  }
  if ((r = dsem_int::check_flag(c))) return r;
  double Jv = 0.0, lr_explicit = 0.0;
  for (double s : s_win) {
    Jv += dt * (A.s2 > 0 ? 100.0 * (s / A.s2) * (1.0 / c->P.re) : 0.0);
    lr_explicit += dt * (A.s2 > 0 ? 100.0 * (s / A.s2) : 0.0);
  }
  // ---- reverse sweep
  CKA(cudaMemsetAsync(A.b.lq, 0, bq, c->st));
  CKA(cudaMemsetAsync(A.b.lg, 0, bq, c->st));
  CKA(cudaMemsetAsync(A.b.lr, 0, sizeof(double), c->st));
  CKA(cudaMemsetAsync(A.b.lrp, 0, (size_t)c->ngrid * sizeof(double), c->st));  // per element, summed over stages
  if (window > 0) {
    if (snapshots == 0) {
      // Every reverse step launches the same kernels with other stage pointers:
      // after the first (eager) step, each step is captured and replayed as a
      // CUDA graph, one executable graph per kind of step (inside or outside
      // the objective's window) updated in place with the new pointers.
      cudaGraphExec_t gx[2] = {nullptr, nullptr};
      auto drop = [&]() {
        for (auto &x : gx)
          if (x) cudaGraphExecDestroy(x);
      };
      for (int n = nsteps - 1; n >= 0; --n) {
        std::vector<double *> st, qf;
        for (int k = 0; k < kord; ++k) {
          st.push_back(A.b.stages + ((size_t)n * kord + k) * nq);
          if (A.b.traces) qf.push_back(A.b.traces + ((size_t)n * kord + k) * nf);
        }
        double *const *qfp = qf.empty() ? nullptr : qf.data();
        const double *qend = n + 1 < nsteps ? A.b.stages + ((size_t)(n + 1) * kord) * nq : c->JQ;
        // the previous step's last stage (entropy viscosity)
        const double *qprev = n > 0 ? A.b.stages + ((size_t)(n - 1) * kord + kord - 1) * nq : nullptr;
        const double *qfprev = (n > 0 && A.b.traces) ? A.b.traces + ((size_t)(n - 1) * kord + kord - 1) * nf : nullptr;
        // the gradients step n's last stage saved: kept by the forward sweep, or with
        // entropy viscosity the group's EVB (the forward sweep's last step, then
        // each reverse step's recomputation for the step before it)
        const double *evb = A.visc ? EVB_GROUPS
                                 : ((A.in_window(n) && A.b.evbw) ? A.b.evbw + (size_t)(n - (nsteps - window)) * nevb
                                                                 : nullptr);
        if (n == nsteps - 1 || (A.visc && n == 0)) {  // launch sequences of their own: eager
          if ((r = reverse_step(A, n, st.data(), qend, qfp, qprev, qfprev, evb))) return drop(), r;
          continue;
        }
        r = replay(c, &gx[A.in_window(n) ? 1 : 0],
                   [&] { return reverse_step(A, n, st.data(), qend, qfp, qprev, qfprev, evb); });
        if (r) return drop(), r;
      }
      drop();
    } else {
      CKA(cudaMemcpyAsync(A.b.slots[0], A.b.q0, bq, cudaMemcpyDeviceToDevice, c->st));
      if (A.visc) {  // the first step's viscosity reads the gradients from before the run
        if (A.ev_valid0) CKA(cudaMemcpyAsync(A.b.slot_evb[0], A.b.evb0, evb_bytes(A), cudaMemcpyDeviceToDevice, c->st));
        A.b.slot_valid[0] = A.ev_valid0 ? 1 : 0;
      }
      if (seg_k) {
        // segments, last first: recompute each from its snapshot into the stash, then reverse it
        cudaGraphExec_t gf[2] = {nullptr, nullptr}, gr[2] = {nullptr, nullptr};
        auto drop = [&]() {
          for (auto *x : {&gf[0], &gf[1], &gr[0], &gr[1]})
            if (*x) cudaGraphExecDestroy(*x);
        };
        for (int j = nseg - 1; j >= 0; --j) {
          const int b = j * seg_k, e = std::min(nsteps, b + seg_k);
          if (j < nseg - 1 &&
              ((r = load_slot(A, j)) || (r = keep_prev(A)) || (r = seg_forward(A, b, e, nullptr, gf))))
            return drop(), r;
          if ((r = seg_reverse(A, b, e, j == nseg - 1, gr))) return drop(), r;
        }
        drop();
      } else if ((r = revolve_spine(A, 0, nsteps, 0, 1))) {
        return r;
      }
    }
  }
  k_sum_into<<<1, 256, 0, c->st>>>(A.b.lrp, c->ngrid, A.b.lr);  // dJ/d(1/Re) of the volume terms
  CKA(cudaGetLastError());
  if (nbpt) {  // ... and of the external viscous fluxes of inflow and outflow faces
    k_sum_into<<<1, 256, 0, c->st>>>(A.b.lrb, (int)nbpt, A.b.lr);
    CKA(cudaGetLastError());
  }
  CKA(cudaEventRecord(e1, c->st));
  CKA(cudaEventSynchronize(e1));
  float t = 0.f;
  CKA(cudaEventElapsedTime(&t, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  double lr_dev = 0.0;
  CKA(cudaMemcpy(&lr_dev, A.b.lr, sizeof(double), cudaMemcpyDeviceToHost));
  if (J) *J = Jv;
  if (dJdinvRe) *dJdinvRe = lr_dev + lr_explicit;
  if (ms) *ms = t;
  if (dJdQ0 && (r = dsem_int::unpack_state(c, A.b.lq, dJdQ0, ldx))) return r;
  // restore the initial state
  CKA(cudaMemcpyAsync(c->JQ, A.b.q0, bq, cudaMemcpyDeviceToDevice, c->st));
  if ((r = dsem_int::traces(c))) return r;
  c->grad_valid = false;
  c->ev_grad_valid = false;
  c->last_ms = t;
  c->last_launches = A.launches;
  CKA(cudaStreamSynchronize(c->st));
  return DSEM_OK;
}
