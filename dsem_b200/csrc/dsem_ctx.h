// dsem_ctx.h -- the library's context (opaque behind include/dsem_gpu.h) and
// the per-order dispatch helper, shared by the translation units of the C-ABI.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <type_traits>
#include <vector>

#include "dsem_launch.h"
#include "dsem_stage.cuh"

namespace dsem {

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

struct Group {
  int G = 0, nel = 0;
  bool diag = true;
  long long e0 = 0;  // first internal element
  long long q0 = 0;  // offset of the group's state (doubles)
  long long f0 = 0;  // offset of the group's face slots (doubles)
  double *jac = nullptr, *gg = nullptr, *gm = nullptr, *hd = nullptr;
  double *muhg = nullptr, *EVB = nullptr, *kew = nullptr;
  double *nuhg = nullptr;  // Smagorinsky viscosity at Gauss points (LES on)
  long long l0 = 0;        // offset of the group's kept Lobatto arrays in dsem_ctx::QLB (doubles)
  double *sens = nullptr;  // [elem][2][G^3] Ducros and density sensors (Smagorinsky sensors on)
  int *int2ext = nullptr;  // device: caller element id of each group element
  int *ecase = nullptr;    // device: case of each group element
  MortarC *fmc = nullptr;  // device: [elem][6] mortar of each face, bit 8 of flags on a slave side (fuse_vis)
  std::vector<int> case_lo, case_hi;  // group elements [lo, hi) of each case
};

struct MList {  // conforming mortars of one order
  int G = 0, n = 0;
  MortarC *mc = nullptr;
  double *nh = nullptr, *nrm = nullptr;
};

struct BList {  // boundary mortars (id(2) = 0) of one order
  int G = 0, n = 0;
  MortarB *mb = nullptr;
  double *nh = nullptr, *nrm = nullptr;
  double *qext = nullptr, *fvext = nullptr;  // external mrtr%Q / mrtr%fv (side 2), [n][5][G^2]
  std::vector<int> mortar;                   // caller mortar index of each entry
};

}  // namespace dsem

using dsem::Group;
using dsem::MList;
using dsem::BList;
using dsem::MortarNC;
using dsem::MortarCut;
using dsem::Phys;

struct dsem_ctx {
  int dev = 0;
  cudaStream_t st = nullptr;
  int ngrid = 0, nmort = 0;
  Phys P{};
  int shock = 0, iord = 4, kord = 5;
  int les = 0;                     // static Smagorinsky model (dsem_set_les)
  double les_cs = 0.0, les_numax = 0.0;
  int les_sensors = 0;             // bit 0: shockSensor, bit 1: rhoSensor (dsem_set_les_sensors)
  double ark[5] = {}, brk[5] = {}, crk[5] = {};
  std::vector<Group> groups;
  std::vector<MList> mlists;
  // every element face is one side of one conforming mortar: dsem_step's update kernel
  // averages the viscous face fluxes itself (Group::fmc) and no k_face_vis runs
  bool fuse_vis = false;
  int vol_variant[dsem::GMAX + 1] = {};  // launch shape of the volume kernel per order G (dsem_autotune)
  std::vector<BList> blists;  // boundary faces; their conditions need dsem_set_boundary first
  int nbnd = 0;
  bool bnd_need_twall = false, bnd_need_ext = false, bnd_twall_set = false, bnd_ext_set = false;
  double twall = 0.0;
  MortarNC *nc = nullptr;  // p-nonconforming mortars
  int nnc = 0;
  double *nc_nh = nullptr, *nc_nrm = nullptr, *nc_mats = nullptr;
  std::vector<int> ext_group, ext_k;  // caller element -> (group, index in group)
  double *JQ = nullptr, *gQ = nullptr, *QTI = nullptr, *QF = nullptr, *FF = nullptr, *VF = nullptr;
  double *Qt = nullptr, *stage = nullptr, *part = nullptr;
  size_t nq = 0, nface = 0, nstage = 0;
  int stage_ldx = 0;
  int *flag = nullptr;
  bool traces_valid = false;
  bool grad_valid = false;     // EVB holds the Q gradients of the last Fluxes call
  bool ev_grad_valid = false;  // ... and the temperature gradients (EV)
  int keep_grad = 0;
  // Lobatto arrays of the last stage (DSEM's d%Qlgg/Qglg/Qggl) kept for the restart file
  double *QLB = nullptr;  // [elem][3][5][L*G^2] per group at Group::l0
  bool keep_lob = false;  // the last stage of every step stores them (dsem_keep_lobatto)
  bool lob_valid = false; // QLB holds the arrays of the last stage run
  int adj_scheme = 0;     // dsem_adjoint with snapshots > 0: DSEM_ADJ_REVOLVE or DSEM_ADJ_SEGMENTS
  cudaGraphExec_t gexec = nullptr;
  int graph_key = -1;
  long long graph_launches = 0;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  double last_ms = 0.0;
  long long last_launches = 0;
  std::string err;
  std::vector<double> host_part;
  // ensemble: independent cases sharing the launches (a single case is an ensemble of one)
  int ncase = 1;
  std::vector<int> case_el0;         // first caller element of each case (+ total)
  std::vector<double> case_re, case_dt, case_prestep;
  double *d_rec = nullptr;           // device: per case {re, 1/re}
  double *d_dtc = nullptr;           // device: per case dt of the current call
  // order groups run as parallel branches of the stream (and of the captured graph)
  std::vector<cudaStream_t> aux;
  std::vector<cudaEvent_t> ev_join;
  cudaEvent_t ev_fork = nullptr;
  // sharding: mortars whose other side lives on another shard; the remote
  // face data arrive in `ghost` (one 5 x G^2 block per cut mortar), the local
  // faces leave through `send` (same order)
  int ncut = 0, cut_G = 0;
  dsem::MortarCut *cut = nullptr;
  double *cut_nh = nullptr, *cut_nrm = nullptr;
  long long *pack_src = nullptr;
  double *send = nullptr, *ghost = nullptr;
};

// error text of calls made without a context (read by dsem_last_error(NULL))
void dsem_set_thread_error(const std::string &msg);

// Internal entry points of the API translation unit used by the adjoint.
namespace dsem_int {
int fail(dsem_ctx *c, int code, const std::string &msg);
int stage(dsem_ctx *c, int kk, bool save);  // one RK stage on c->JQ (eager launches)
int traces(dsem_ctx *c);                    // face traces of c->JQ
int ev(dsem_ctx *c, const double *jq = nullptr);  // entropy viscosity of jq (null: c->JQ; valid: c->ev_grad_valid)
int les(dsem_ctx *c, const double *jq = nullptr);  // Smagorinsky viscosity of jq (null: c->JQ; valid: c->grad_valid)
struct StageIO {
  double *jq_in;        // stage input state (read only)
  const double *qf_in;  // its raw face traces (read only)
  double *jq_out, *qf_out;  // updated state and its raw face traces
  double *evb;              // where a saving stage puts its gradients (null: the group's EVB)
};
int stage_io(dsem_ctx *c, int kk, bool save, const StageIO &io);  // out-of-place stage (one group, periodic)
int set_dt(dsem_ctx *c, const double *dt);
int unpack_state(dsem_ctx *c, const double *dev, double *host, int ldx);
int check_flag(dsem_ctx *c);
// kept Lobatto arrays (dsem_keep_lobatto): per caller element [3][5][L*G^2] at lob_offsets()[e]
std::vector<long long> lob_offsets(const dsem_ctx *c);
int lob_download(dsem_ctx *c, double *host);
int lob_upload_grad(dsem_ctx *c, const double *host);
void grad_invalidate(dsem_ctx *c);
// enstrophy sums of the last saved gradients with the state jq (null: c->JQ)
int eps_sums(dsem_ctx *c, double *s, double *s2, const double *jq = nullptr);
// the same in two halves: per-element partials into device memory part
// ([elements][5], no sync; gradients from evb, null: the group's EVB, one
// group only when given), then the sums from a host copy of them
int eps_enqueue(dsem_ctx *c, const double *jq, double *part, const double *evb = nullptr);
void eps_reduce(const dsem_ctx *c, const double *part, double *s, double *s2);
}  // namespace dsem_int
