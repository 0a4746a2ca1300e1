// dsem_oracle.cpp -- CPU oracle (TEST INFRASTRUCTURE, the checker) for the
// DSEM right-hand side + low-storage Runge-Kutta stage.
//
// Restates, routine by routine, the Fortran of mranjb2/DSEM (paths relative
// to the DSEM source tree).  Nothing here is product code: the CUDA library
// never links it.  Parity against DSEM itself is unpinned (no golden vectors,
// no Fortran toolchain); known-answer tests in tests/ pin the restatement.
//
// Evaluation order (the contract shared with the CUDA kernels, so that the
// two agree bit for bit on the same inputs):
//  * every small contraction  y_i = sum_k A_ik x_k  is an FMA chain in
//    increasing k:  acc = A_i0*x_0; acc = fma(A_ik, x_k, acc) ...
//  * pointwise physics is evaluated in DSEM's expression order without
//    contraction (this file is compiled with -ffp-contract=off).
//  * the flux divergence adds interior Lobatto terms first and the two face
//    terms of each direction afterwards (see update_element).
// DSEM's Fortran sums the same terms left to right without FMA; the two
// orders differ by rounding only.
#include "dsem_oracle.h"

#include <algorithm>
#include <array>
#include <cfloat>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr double PI = 3.141592653589793238462643;  // initializationsc2.f90:25
constexpr int NV = 5;
constexpr int NMX = 16;  // stride of mortar-space scratch arrays

// ------------------------------------------------------------------ scalars
inline double fmac(double a, double b, double c) { return std::fma(a, b, c); }
inline std::complex<double> fmac(double a, std::complex<double> b, std::complex<double> c) {
  return a * b + c;
}
inline double re_(double x) { return x; }
inline double re_(std::complex<double> x) { return x.real(); }
template <class T> inline T rabs(T x) { return re_(x) < 0 ? -x : x; }
template <class T> inline T rmax(T a, T b) { return re_(a) >= re_(b) ? a : b; }
template <class T> inline T rmin(T a, T b) { return re_(a) <= re_(b) ? a : b; }
template <class T> inline bool rfinite(T x) { return std::isfinite(re_(x)) && std::isfinite(std::imag(std::complex<double>(x))); }

// ------------------------------------------------ polynomials: baselib.f90:18-80
double polyn(int k, double x, int n, const double *z) {
  double p;
  if (k == 0) {
    p = (x - z[1]) / (z[0] - z[1]);
    for (int j = 2; j < n; ++j) p = p * (x - z[j]) / (z[0] - z[j]);
  } else {
    p = (x - z[0]) / (z[k] - z[0]);
    for (int j = 1; j < k; ++j) p = p * (x - z[j]) / (z[k] - z[j]);
    for (int j = k + 1; j < n; ++j) p = p * (x - z[j]) / (z[k] - z[j]);
  }
  return p;
}

double polynder(int k, double x, int n, const double *z) {
  double hp = 0.0;
  for (int l = 0; l < n; ++l) {
    if (l == k) continue;
    double poly = 1.0;
    for (int m = 0; m < n; ++m) {
      if (m == l || m == k) continue;
      poly = poly * (x - z[m]) / (z[k] - z[m]);
    }
    hp = hp + poly / (z[k] - z[l]);
  }
  return hp;
}

// --------------------------------------------- points: stac3m_geomLib.f90:7-75
void lobatto_points(int L, double *cx) {
  const int na = L - 1;
  for (int n = 0; n < L; ++n) {
    double xx = std::cos((double)n * PI / (double)na);
    cx[n] = 0.5 * (1.0 - xx);
  }
}
void gauss_points(int G, double *cxg) {
  for (int n = 1; n <= G; ++n) {
    double xx = std::cos((2.0 * n - 1.0) * PI / (2.0 * ((double)G - 1.0) + 2.0));
    cxg[n - 1] = 0.5 * (1.0 - xx);
  }
}

// ------------------------------------- operators: matrices.f90:144-207
struct Ops {
  int G = 0, L = 0;
  std::vector<double> cx, cxg, dmx /*[G][L]*/, bx /*[L][G]*/;
};
void build_ops(int G, Ops &o) {
  o.G = G;
  o.L = G + 1;
  const int L = o.L;
  o.cx.resize(L);
  o.cxg.resize(G);
  lobatto_points(L, o.cx.data());
  gauss_points(G, o.cxg.data());
  o.dmx.assign(G * L, 0.0);
  o.bx.assign(L * G, 0.0);
  const double eps = DBL_EPSILON;  // 3DDriver_parfmdf.f90:126
  for (int k = 0; k < G; ++k) {   // dermat (matrices.f90:144-178)
    double sum = 0.0;
    for (int j = 0; j < L; ++j) {
      if (j == k) continue;
      double b = polynder(j, o.cxg[k], L, o.cx.data());
      if (std::fabs(b) < eps) b = 0.0;
      o.dmx[k * L + j] = b;
      sum = sum - b;
      o.dmx[k * L + k] = sum;
    }
  }
  for (int n = 0; n < L; ++n)   // intrpmat (matrices.f90:185-207)
    for (int j = 0; j < G; ++j) o.bx[n * G + j] = polyn(j, o.cx[n], G, o.cxg.data());
}
const Ops &ops_for(int G) {
  // built once (thread-safe static initialisation), read-only afterwards
  static const std::vector<Ops> cache = [] {
    std::vector<Ops> v(17);
    for (int g = 2; g <= 16; ++g) build_ops(g, v[g]);
    return v;
  }();
  return cache.at(G);
}

// ------------------ Gauss-Legendre nodes/weights on [-1,1] (gaussq, legendre_routines.f90:98)
// Newton iteration on the three-term recurrence; nodes ascending.
void gauss_legendre(int n, double *x, double *w) {
  for (int i = 0; i < n; ++i) {
    double z = std::cos(PI * (i + 0.75) / (n + 0.5));
    double pp = 0.0;
    for (int it = 0; it < 100; ++it) {
      double p1 = 1.0, p2 = 0.0;
      for (int j = 0; j < n; ++j) {
        double p3 = p2;
        p2 = p1;
        p1 = ((2.0 * j + 1.0) * z * p2 - j * p3) / (j + 1.0);
      }
      pp = n * (z * p1 - p2) / (z * z - 1.0);
      double dz = p1 / pp;
      z -= dz;
      if (std::fabs(dz) < 1e-17) break;
    }
    x[n - 1 - i] = z;
    w[n - 1 - i] = 2.0 / ((1.0 - z * z) * pp * pp);
  }
}

// ------------------- mortar projections: mortarLib.f90:242-420, LU :456-692
void lu_solve_matrix(int n, std::vector<double> a, double *rhs /*[n][ncol] col-major*/, int ncol) {
  std::vector<int> piv(n);
  for (int k = 0; k < n; ++k) {
    int p = k;
    for (int i = k + 1; i < n; ++i)
      if (std::fabs(a[i + n * k]) > std::fabs(a[p + n * k])) p = i;
    piv[k] = p;
    if (p != k)
      for (int j = 0; j < n; ++j) std::swap(a[k + n * j], a[p + n * j]);
    for (int i = k + 1; i < n; ++i) {
      a[i + n * k] /= a[k + n * k];
      for (int j = k + 1; j < n; ++j) a[i + n * j] -= a[i + n * k] * a[k + n * j];
    }
  }
  for (int c = 0; c < ncol; ++c) {
    double *b = rhs + (size_t)n * c;
    for (int k = 0; k < n; ++k) {
      std::swap(b[k], b[piv[k]]);
      for (int i = k + 1; i < n; ++i) b[i] -= a[i + n * k] * b[k];
    }
    for (int k = n - 1; k >= 0; --k) {
      for (int j = k + 1; j < n; ++j) b[k] -= a[k + n * j] * b[j];
      b[k] /= a[k + n * k];
    }
  }
}
// compute_pmat: projection from nodes cxin (ni) to nodes cxo (no); out [no][ni]
void compute_pmat(const double *cxin, int ni, const double *cxo, int no, double *pmat) {
  std::vector<double> xg(std::max(ni, no)), wg(std::max(ni, no));
  gauss_legendre(no, xg.data(), wg.data());
  std::vector<double> bm(no * no);
  for (int i = 0; i < no; ++i)
    for (int j = 0; j < no; ++j) {
      double s = 0.0;
      for (int k = 0; k < no; ++k) {
        double hj = polyn(j, 0.5 * (xg[k] + 1.0), no, cxo);
        double hi = polyn(i, 0.5 * (xg[k] + 1.0), no, cxo);
        s = s + 0.5 * wg[k] * hi * hj;
      }
      bm[i + no * j] = s;
    }
  const int ncc = std::max(ni, no);
  gauss_legendre(ncc, xg.data(), wg.data());
  std::vector<double> am(no * ni);
  for (int i = 0; i < no; ++i)
    for (int j = 0; j < ni; ++j) {
      double s = 0.0;
      for (int k = 0; k < ncc; ++k) {
        double xi = 0.5 * (xg[k] + 1.0);
        double hin = polyn(j, xi, ni, cxin);
        double hout = polyn(i, xi, no, cxo);
        s = s + 0.5 * wg[k] * hin * hout;
      }
      am[i + no * j] = s;
    }
  lu_solve_matrix(no, bm, am.data(), ni);
  const double eps = 100 * DBL_EPSILON;
  for (int i = 0; i < no; ++i)
    for (int j = 0; j < ni; ++j) {
      double v = am[i + no * j];
      pmat[i * ni + j] = std::fabs(v) <= eps ? 0.0 : v;
    }
}

// --------------------------------------------- hex8 geometry: GeomLib3D.f90
void hex8_map(const double c[8][3], const double cx[3], double x[3]) {  // :60-85
  for (int j = 0; j < 3; ++j)
    x[j] = c[0][j] * (1.0 - cx[0]) * (1.0 - cx[1]) * (1.0 - cx[2]) +
           c[1][j] * cx[0] * (1.0 - cx[1]) * (1.0 - cx[2]) +
           c[2][j] * cx[0] * cx[1] * (1.0 - cx[2]) +
           c[3][j] * (1.0 - cx[0]) * cx[1] * (1.0 - cx[2]) +
           c[4][j] * (1.0 - cx[0]) * (1.0 - cx[1]) * cx[2] +
           c[5][j] * cx[0] * (1.0 - cx[1]) * cx[2] +
           c[6][j] * cx[0] * cx[1] * cx[2] +
           c[7][j] * (1.0 - cx[0]) * cx[1] * cx[2];
}
void grad_hex8_map(const double c[8][3], const double cx[3], double g[3][3]) {  // :99-146
  for (int i = 0; i < 3; ++i) {
    g[i][0] = -c[0][i] * (1.0 - cx[1]) * (1.0 - cx[2]) + c[1][i] * (1.0 - cx[1]) * (1.0 - cx[2]) +
              c[2][i] * cx[1] * (1.0 - cx[2]) - c[3][i] * cx[1] * (1.0 - cx[2]) -
              c[4][i] * (1.0 - cx[1]) * cx[2] + c[5][i] * (1.0 - cx[1]) * cx[2] +
              c[6][i] * cx[1] * cx[2] - c[7][i] * cx[1] * cx[2];
    g[i][1] = -c[0][i] * (1.0 - cx[0]) * (1.0 - cx[2]) - c[1][i] * cx[0] * (1.0 - cx[2]) +
              c[2][i] * cx[0] * (1.0 - cx[2]) + c[3][i] * (1.0 - cx[0]) * (1.0 - cx[2]) -
              c[4][i] * (1.0 - cx[0]) * cx[2] - c[5][i] * cx[0] * cx[2] +
              c[6][i] * cx[0] * cx[2] + c[7][i] * (1.0 - cx[0]) * cx[2];
    g[i][2] = -c[0][i] * (1.0 - cx[0]) * (1.0 - cx[1]) - c[1][i] * cx[0] * (1.0 - cx[1]) -
              c[2][i] * cx[0] * cx[1] - c[3][i] * (1.0 - cx[0]) * cx[1] +
              c[4][i] * (1.0 - cx[0]) * (1.0 - cx[1]) + c[5][i] * cx[0] * (1.0 - cx[1]) +
              c[6][i] * cx[0] * cx[1] + c[7][i] * (1.0 - cx[0]) * cx[1];
  }
}
// Invert_Metric_Tensor (GeomLib3D.f90:685-734): gc[i][j] = dX_i/dx_j
void invert_metric(const double gx[3][3], double gc[3][3], double &J) {
  const double small = 100 * DBL_EPSILON;
  J = gx[0][0] * gx[1][1] * gx[2][2] - gx[0][1] * gx[1][0] * gx[2][2] -
      gx[0][0] * gx[1][2] * gx[2][1] + gx[0][2] * gx[1][0] * gx[2][1] +
      gx[0][1] * gx[1][2] * gx[2][0] - gx[0][2] * gx[1][1] * gx[2][0];
  gc[0][0] = (gx[1][1] * gx[2][2] - gx[1][2] * gx[2][1]) / J;
  gc[1][0] = (-gx[1][0] * gx[2][2] + gx[1][2] * gx[2][0]) / J;
  gc[2][0] = (gx[1][0] * gx[2][1] - gx[2][0] * gx[1][1]) / J;
  gc[0][1] = (-gx[0][1] * gx[2][2] + gx[0][2] * gx[2][1]) / J;
  gc[1][1] = (gx[0][0] * gx[2][2] - gx[0][2] * gx[2][0]) / J;
  gc[2][1] = (-gx[0][0] * gx[2][1] + gx[0][1] * gx[2][0]) / J;
  gc[0][2] = (gx[0][1] * gx[1][2] - gx[1][1] * gx[0][2]) / J;
  gc[1][2] = (-gx[0][0] * gx[1][2] + gx[0][2] * gx[1][0]) / J;
  gc[2][2] = (gx[0][0] * gx[1][1] - gx[0][1] * gx[1][0]) / J;
  for (int m = 0; m < 3; ++m)
    for (int n = 0; n < 3; ++n)
      if (std::fabs(gc[n][m]) <= small) gc[n][m] = 0.0;
}

// ------------------------------------------------------------ data types
template <class T> struct Elem {
  int G = 0, L = 0;
  double corner[8][3] = {};
  int node[8] = {};
  int mort[6] = {-1, -1, -1, -1, -1, -1};
  int mside[6] = {0, 0, 0, 0, 0, 0};  // 1 master, 2 slave
  int orientation[6] = {};
  bool boundary[6] = {};
  int bcond[6] = {};  // d%bcond as BC_* codes (faces without a neighbour)
  std::vector<double> jacob, gmetg, gmet[3], xg, hdelta;
  std::vector<T> Q, gQ, QL[3], F[3], R[3], muhg, muh[3], nutg, nut[3];
  std::vector<T> ducros, rhos;  // d%ducros, d%rhoSensor at the Gauss points (RHS.f90:180-181; zero_domain: 0)
  size_t ng() const { return (size_t)G * G * G; }
  size_t nl() const { return (size_t)L * G * G; }
};

template <class T> struct Mortar {
  int id[2] = {-1, -1}, iface[2] = {0, 0};
  int len[2][2] = {};  // len[dir][side]
  int lenm[2] = {};
  int orient = 0, sign = 1, nsign = 1;
  bool conf[2][2] = {{true, true}, {true, true}};  // conf[dir][side]
  std::vector<double> n_hat, norm;                 // [j*NMX+i]*3, [j*NMX+i]
  std::vector<double> P[2][2], Rm[2][2];           // [side][dir]
  int pin[2][2] = {};                              // input extent of P[side][dir]
  std::vector<T> Qm[2], fv[2];                     // [v][j*NMX+i]
  int bc = 0;                                      // boundary mortar (id(2) = 0): bcond of the master face
  std::vector<double> Qx, fvx;                     // external mrtr%Q(:,:,:,2), mrtr%fv(:,:,:,2): [v][j*NMX+i]
};

// boundary condition codes (the CHARACTER d%bcond values of the problem file)
enum { BC_INTERFACE = 0, BC_WALLADIAB = 1, BC_WALLISOTH = 2, BC_INFLOW = 3, BC_OUTFLOW = 4 };

template <class T> struct Case {
  std::vector<Elem<T>> el;
  std::vector<Mortar<T>> mo;
  double gamma = 1.4, re = 1600.0, pr = 0.72, mach = 1.0, cmu = 0.0, mumax = 0.0;
  bool shock = false, ducros = false;
  bool les = false;               // static Smagorinsky (staticSmag.f90)
  bool shock_sensor = false, rho_sensor = false;  // shockSensor, rhoSensor (input_lib.f90:163-164)
  double cs = 0.0, numax = 0.0;  // C_s, numax
  int iord = 4, kord = 5;
  double ark[5] = {}, brk[5] = {}, crk[5] = {};
  bool ql_valid = false;
  double prestep = 0.0;
  double twall = 0.0;  // wall temperature of isothermal walls (MODULE physics)
};

// -------------------------------------------------- rkcoefs (baselib.f90:86-160)
template <class T> void rkcoefs(Case<T> &c, int iord) {
  for (int i = 0; i < 5; ++i) c.ark[i] = c.brk[i] = c.crk[i] = 0.0;
  c.iord = iord;
  switch (iord) {
    case 1:
      c.kord = 1;
      c.crk[0] = 1.0;
      break;
    case 2:
      c.kord = 2;
      c.ark[1] = -1.0;
      c.brk[1] = 1.0;
      c.crk[0] = 1.0;
      c.crk[1] = 0.5;
      break;
    case 3:
      c.kord = 3;
      c.ark[1] = -5.0 / 9.0;
      c.ark[2] = -153.0 / 128.0;
      c.brk[1] = 1.0 / 3.0;
      c.brk[2] = 3.0 / 4.0;
      c.crk[0] = 1.0 / 3.0;
      c.crk[1] = 15.0 / 16.0;
      c.crk[2] = 8.0 / 15.0;
      break;
    default:
      c.kord = 5;
      c.ark[1] = -0.4178904745;
      c.ark[2] = -1.192151694643;
      c.ark[3] = -1.697784692471;
      c.ark[4] = -1.514183444257;
      c.brk[1] = 0.1496590219993;
      c.brk[2] = 0.3704009573644;
      c.brk[3] = 0.6222557631345;
      c.brk[4] = 0.9582821306748;
      c.crk[0] = 0.1496590219993;
      c.crk[1] = 0.3792103129999;
      c.crk[2] = 0.8229550293869;
      c.crk[3] = 0.6994504559488;
      c.crk[4] = 0.1530572479681;
      break;
  }
}

// ---------------------------------------------------- grid index helpers
// Gauss (n,m,l): n + G*(m + G*l).  Grid d=0 (lgg) n<L: n + L*(m + G*l);
// d=1 (glg) m<L: n + G*(m + L*l); d=2 (ggl) l<L: n + G*(m + G*l).
inline size_t gidx(int G, int n, int m, int l) { return n + (size_t)G * (m + (size_t)G * l); }
inline size_t lidx(int d, int G, int L, int n, int m, int l) {
  if (d == 0) return n + (size_t)L * (m + (size_t)G * l);
  if (d == 1) return n + (size_t)G * (m + (size_t)L * l);
  return n + (size_t)G * (m + (size_t)G * l);
}
// face (1..6) point (i,j) -> (grid, n, m, l)   (send_q.f90:491-764)
inline void face_point(int face, int G, int L, int i, int j, int &d, int &n, int &m, int &l) {
  (void)G;
  switch (face) {
    case 1: d = 1; n = i; m = 0; l = j; break;
    case 2: d = 1; n = i; m = L - 1; l = j; break;
    case 3: d = 2; n = i; m = j; l = 0; break;
    case 5: d = 2; n = i; m = j; l = L - 1; break;
    case 4: d = 0; n = L - 1; m = i; l = j; break;
    default: d = 0; n = 0; m = i; l = j; break;
  }
}
template <class T> inline T &face_ref(std::vector<T> *arr, const Elem<T> &E, int face, int i, int j, int v) {
  int d, n, m, l;
  face_point(face, E.G, E.L, i, j, d, n, m, l);
  return arr[d][(size_t)v * E.nl() + lidx(d, E.G, E.L, n, m, l)];
}

// ----------------------------------------------------- physics: PhysLib.f90
template <class T> void euler_fluxes(const T *Q, double gamma, T *f, T *g, T *h) {  // :17-124
  T rho = Q[0], rhou = Q[1], rhov = Q[2], rhow = Q[3], rhoe = Q[4];
  T u = rhou / rho, v = rhov / rho, w = rhow / rho;
  T p = (gamma - 1.0) * (rhoe - 0.5 * rho * (u * u + v * v + w * w));
  f[0] = rhou; f[1] = p + rhou * u; f[2] = rhou * v; f[3] = rhou * w; f[4] = u * (rhoe + p);
  g[0] = rhov; g[1] = rhou * v; g[2] = p + rhov * v; g[3] = rhow * v; g[4] = v * (rhoe + p);
  h[0] = rhow; h[1] = rhou * w; h[2] = rhov * w; h[3] = p + rhow * w; h[4] = w * (rhoe + p);
}

// Roe flux with entropy fix: riemann (PhysLib.f90:231-320)
template <class T> void riemann(const double *nh, double ds, const T *Ql, const T *Qr, double gamma, T *flux) {
  T rho = Ql[0], rhou = Ql[1], rhov = Ql[2], rhow = Ql[3], rhoe = Ql[4];
  T rhon = Qr[0], rhoun = Qr[1], rhovn = Qr[2], rhown = Qr[3], rhoen = Qr[4];
  T ul = rhou / rho, vl = rhov / rho, wl = rhow / rho;
  T pleft = (gamma - 1.0) * (rhoe - 0.5 / rho * (rhou * rhou + rhov * rhov + rhow * rhow));
  T ur = rhoun / rhon, vr = rhovn / rhon, wr = rhown / rhon;
  T pright = (gamma - 1.0) * (rhoen - 0.5 / rhon * (rhoun * rhoun + rhovn * rhovn + rhown * rhown));
  T ql = nh[0] * ul + nh[1] * vl + nh[2] * wl;
  T qr = nh[0] * ur + nh[1] * vr + nh[2] * wr;
  T hl = 0.5 * (ul * ul + vl * vl + wl * wl) + gamma / (gamma - 1.0) * pleft / rho;
  T hr = 0.5 * (ur * ur + vr * vr + wr * wr) + gamma / (gamma - 1.0) * pright / rhon;
  T rtd = std::sqrt(rho * rhon);
  T betal = rho / (rho + rtd);
  T betar = 1.0 - betal;
  T utd = betal * ul + betar * ur;
  T vtd = betal * vl + betar * vr;
  T wtd = betal * wl + betar * wr;
  T htd = betal * hl + betar * hr;
  T atd2 = (gamma - 1.0) * (htd - 0.5 * (utd * utd + vtd * vtd + wtd * wtd));
  T atd = std::sqrt(atd2);
  T qtd = utd * nh[0] + vtd * nh[1] + wtd * nh[2];
  if (re_(qtd) >= 0.0) {
    T dw1 = 0.5 * ((pright - pleft) / atd2 - (qr - ql) * rtd / atd);
    T sp1 = qtd - atd;
    T sp1m = rmin(sp1, T(0.0));
    T hd1m = ((gamma + 1.0) / 4.0 * atd / rtd) * dw1;
    T eta1 = rmax(-rabs(sp1) - hd1m, T(0.0));
    T udw1 = dw1 * (sp1m - 0.5 * eta1);
    T rql = rho * ql;
    flux[0] = ds * (rql + udw1);
    flux[1] = ds * (rql * ul + pleft * nh[0] + udw1 * (utd - atd * nh[0]));
    flux[2] = ds * (rql * vl + pleft * nh[1] + udw1 * (vtd - atd * nh[1]));
    flux[3] = ds * (rql * wl + pleft * nh[2] + udw1 * (wtd - atd * nh[2]));
    flux[4] = ds * (rql * hl + udw1 * (htd - qtd * atd));
  } else {
    T dw4 = 0.5 * ((pright - pleft) / atd2 + (qr - ql) * rtd / atd);
    T sp4 = qtd + atd;
    T sp4p = rmax(sp4, T(0.0));
    T hd4 = ((gamma + 1.0) / 4.0 * atd / rtd) * dw4;
    T eta4 = rmax(-rabs(sp4) + hd4, T(0.0));
    T udw4 = dw4 * (sp4p + 0.5 * eta4);
    T rqr = rhon * qr;
    flux[0] = ds * (rqr - udw4);
    flux[1] = ds * (rqr * ur + pright * nh[0] - udw4 * (utd + atd * nh[0]));
    flux[2] = ds * (rqr * vr + pright * nh[1] - udw4 * (vtd + atd * nh[1]));
    flux[3] = ds * (rqr * wr + pright * nh[2] - udw4 * (wtd + atd * nh[2]));
    flux[4] = ds * (rqr * hr - udw4 * (htd + qtd * atd));
  }
}

// x/y/z_vis_flux (PhysLib.f90:419-583); the three share the same primitive
// quantities, so they are evaluated once per point (identical arithmetic).
template <class T>
void vis_fluxes(const T *Q, const T *Qx, const T *Qy, const T *Qz, T amu, double gamma, double pr,
                double mach, T *f, T *g, T *h) {
  T rho = Q[0], rhou = Q[1], rhov = Q[2], rhow = Q[3], rhoe = Q[4];
  T u = rhou / rho, v = rhov / rho, w = rhow / rho;
  T p = (gamma - 1.0) * (rhoe - 0.5 * rho * (u * u + v * v + w * w));
  T ux = (Qx[1] - u * Qx[0]) / rho, uy = (Qy[1] - u * Qy[0]) / rho, uz = (Qz[1] - u * Qz[0]) / rho;
  T vx = (Qx[2] - v * Qx[0]) / rho, vy = (Qy[2] - v * Qy[0]) / rho, vz = (Qz[2] - v * Qz[0]) / rho;
  T wx = (Qx[3] - w * Qx[0]) / rho, wy = (Qy[3] - w * Qy[0]) / rho, wz = (Qz[3] - w * Qz[0]) / rho;
  T px = (gamma - 1.0) * (Qx[4] - 0.5 * Qx[0] * (u * u + v * v + w * w) - rho * (u * ux + v * vx + w * wx));
  T py = (gamma - 1.0) * (Qy[4] - 0.5 * Qy[0] * (u * u + v * v + w * w) - rho * (u * uy + v * vy + w * wy));
  T pz = (gamma - 1.0) * (Qz[4] - 0.5 * Qz[0] * (u * u + v * v + w * w) - rho * (u * uz + v * vz + w * wz));
  T tx = (px - p * Qx[0] / rho) * mach * mach * gamma / rho;
  T ty = (py - p * Qy[0] / rho) * mach * mach * gamma / rho;
  T tz = (pz - p * Qz[0] / rho) * mach * mach * gamma / rho;
  T akappa = 1.0 + (amu - 1.0) * 2.0e-1 / (gamma - 1.0);
  T div = ux + vy + wz;
  T sxy = uy + vx, sxz = wx + uz, syz = wy + vz;
  const double den = pr * mach * mach * (gamma - 1.0);
  f[0] = 0.0;
  f[1] = 2.0 * amu * (ux - div / 3.0);
  f[2] = amu * sxy;
  f[3] = amu * sxz;
  f[4] = u * f[1] + v * f[2] + w * f[3] + akappa * tx / den;
  g[0] = 0.0;
  g[1] = amu * sxy;
  g[2] = 2.0 * amu * (vy - div / 3.0);
  g[3] = amu * syz;
  g[4] = v * g[2] + u * g[1] + w * g[3] + akappa * ty / den;
  h[0] = 0.0;
  h[1] = amu * sxz;
  h[2] = amu * syz;
  h[3] = 2.0 * amu * (wz - div / 3.0);
  h[4] = v * h[2] + u * h[1] + w * h[3] + akappa * tz / den;
}

// ------------------------------------------------ element-level stages
// Contraction along direction d of a 3-D array.
// in: extents (nin along d), out: (nout along d); A[nout][nin].
template <class T>
void contract(int d, const double *A, int nout, int nin, const T *in, const int ein[3], T *out,
              const int eout[3], int k0 = 0, int k1 = -1) {
  // generic index helpers with explicit extents
  if (k1 < 0) k1 = nin;
  int e[3] = {eout[0], eout[1], eout[2]};
  // stride of the input along d, and the input index of (a, b, c) with its d-th index 0
  const size_t sd = d == 0 ? 1 : (d == 1 ? (size_t)ein[0] : (size_t)ein[0] * ein[1]);
  for (int c = 0; c < e[2]; ++c)
    for (int b = 0; b < e[1]; ++b)
      for (int a = 0; a < e[0]; ++a) {
        int ii[3] = {a, b, c};
        const int r = ii[d];
        ii[d] = 0;
        const T *x = in + ii[0] + (size_t)ein[0] * (ii[1] + (size_t)ein[1] * ii[2]);
        const double *row = A + (size_t)r * nin;
        T acc = k0 < k1 ? row[k0] * x[k0 * sd] : T(0.0);
        for (int k = k0 + 1; k < k1; ++k) acc = fmac(row[k], x[k * sd], acc);
        out[a + (size_t)eout[0] * (b + (size_t)eout[1] * c)] = acc;
      }
}
inline void grid_ext(int d, int G, int L, int e[3]) {
  e[0] = e[1] = e[2] = G;
  e[d] = L;
}

// Int_fluxes (fluxesH_newa.f90:221-355): physical Q, Lobatto arrays on the
// three staggered grids (all points), and inviscid interior fluxes.
template <class T> void int_fluxes(Case<T> &c, Elem<T> &E) {
  const Ops &o = ops_for(E.G);
  const int G = E.G, L = E.L;
  const size_t ng = E.ng(), nl = E.nl();
  std::vector<T> q(NV * ng);
  for (int v = 0; v < NV; ++v)
    for (size_t p = 0; p < ng; ++p) q[v * ng + p] = E.Q[v * ng + p] * E.jacob[p];
  const int eg[3] = {G, G, G};
  for (int d = 0; d < 3; ++d) {
    int el[3];
    grid_ext(d, G, L, el);
    E.QL[d].resize(NV * nl);
    E.F[d].assign(NV * nl, T(0.0));
    for (int v = 0; v < NV; ++v) contract(d, o.bx.data(), L, G, &q[v * ng], eg, &E.QL[d][v * nl], el);
    for (int l = 0; l < el[2]; ++l)
      for (int m = 0; m < el[1]; ++m)
        for (int n = 0; n < el[0]; ++n) {
          int idx3[3] = {n, m, l};
          if (idx3[d] == 0 || idx3[d] == L - 1) continue;
          size_t p = lidx(d, G, L, n, m, l);
          T Qv[NV], f[NV], g[NV], h[NV];
          for (int v = 0; v < NV; ++v) Qv[v] = E.QL[d][v * nl + p];
          euler_fluxes(Qv, c.gamma, f, g, h);
          const double *gm = &E.gmet[d][p * 3];
          for (int v = 0; v < NV; ++v) E.F[d][v * nl + p] = gm[0] * f[v] + gm[1] * g[v] + gm[2] * h[v];
        }
  }
}

// ------------------------------------- mortar data movement (mortar_operations.f90)
// mrtr%Q(i,j,v,side) <- face slot  (send_q_to_mortars, send_q.f90:491-764)
template <class T> void gather_face(Case<T> &c, Mortar<T> &M, int side, std::vector<T> *arr, std::vector<T> &dst) {
  Elem<T> &E = c.el[M.id[side]];
  dst.assign(NV * NMX * NMX, T(0.0));
  for (int v = 0; v < NV; ++v)
    for (int j = 0; j < M.len[1][side]; ++j)
      for (int i = 0; i < M.len[0][side]; ++i) dst[v * NMX * NMX + j * NMX + i] = face_ref(arr, E, M.iface[side], i, j, v);
}
// rotate_to_mortar (mortar_operations.f90:461-605)
template <class T> void rotate_to_mortar(const Mortar<T> &M, std::vector<T> &a) {
  if (M.orient == 0) return;
  const int l1 = M.len[0][1], l2 = M.len[1][1];
  std::vector<T> t(a.size(), T(0.0));
  for (int v = 0; v < NV; ++v)
    for (int j = 0; j < l2; ++j)
      for (int i = 0; i < l1; ++i) {
        int ni = i, nj = j;
        switch (M.orient) {
          case 3: ni = i; nj = l2 - 1 - j; break;           // F1B2
          case 2: ni = l1 - 1 - i; nj = l2 - 1 - j; break;  // B1B2
          case 1: ni = l1 - 1 - i; nj = j; break;           // B1F2
          case 4: ni = j; nj = i; break;                    // F2F1
          case 5: ni = l2 - 1 - j; nj = i; break;           // B2F1
          case 6: ni = l2 - 1 - j; nj = l1 - 1 - i; break;  // B2B1
          case 7: ni = j; nj = l1 - 1 - i; break;           // F2B1
        }
        t[v * NMX * NMX + nj * NMX + ni] = a[v * NMX * NMX + j * NMX + i];
      }
  a.swap(t);
}
// rotate_flux_to_face (mortar_operations.f90:616-758)
template <class T> void rotate_to_face(const Mortar<T> &M, std::vector<T> &a) {
  if (M.orient == 0) return;
  const int l1 = M.len[0][1], l2 = M.len[1][1];
  std::vector<T> t(a.size(), T(0.0));
  for (int v = 0; v < NV; ++v)
    for (int j = 0; j < l2; ++j)
      for (int i = 0; i < l1; ++i) {
        int si = i, sj = j;
        switch (M.orient) {
          case 3: si = i; sj = l2 - 1 - j; break;
          case 2: si = l1 - 1 - i; sj = l2 - 1 - j; break;
          case 1: si = l1 - 1 - i; sj = j; break;
          case 4: si = j; sj = i; break;
          case 5: si = l2 - 1 - j; sj = i; break;
          case 6: si = l2 - 1 - j; sj = l1 - 1 - i; break;
          case 7: si = j; sj = l1 - 1 - i; break;
        }
        t[v * NMX * NMX + j * NMX + i] = a[v * NMX * NMX + sj * NMX + si];
      }
  a.swap(t);
}
inline void side_dirs(int orient, int side, int &idir, int &jdir) {
  idir = 0;
  jdir = 1;
  if (side == 1 && orient >= 4) {
    idir = 1;
    jdir = 0;
  }
}
// 1-D projection helper: y[0..nout) = A[nout][nin] x  (FMA chain)
template <class T> void apply1(const double *A, int nout, int nin, const T *x, int xs, T *y, int ys) {
  for (int i = 0; i < nout; ++i) {
    T acc = A[i * nin] * x[0];
    for (int k = 1; k < nin; ++k) acc = fmac(A[i * nin + k], x[(size_t)k * xs], acc);
    y[(size_t)i * ys] = acc;
  }
}
// map_to_mortar_space (mortar_operations.f90:249-344), data in mortar orientation.
template <class T> void map_to_mortar(const Mortar<T> &M, int side, std::vector<T> &a) {
  if (M.conf[0][side] && M.conf[1][side]) return;
  int idir, jdir;
  side_dirs(M.orient, side, idir, jdir);
  const int n1 = M.len[idir][side], n2 = M.len[jdir][side];
  std::vector<T> t(NMX * NMX), y(NMX);
  for (int v = 0; v < NV; ++v) {
    T *A = &a[v * NMX * NMX];
    if (!M.conf[0][side]) {  // direction 1 first (columns j < n2)
      for (int j = 0; j < n2; ++j) apply1(M.P[side][0].data(), M.lenm[0], n1, A + j * NMX, 1, &t[j * NMX], 1);
      for (int j = 0; j < n2; ++j)
        for (int i = 0; i < M.lenm[0]; ++i) A[j * NMX + i] = t[j * NMX + i];
    }
    const int m1 = M.conf[0][side] ? n1 : M.lenm[0];
    if (!M.conf[1][side]) {
      for (int i = 0; i < m1; ++i) {
        apply1(M.P[side][1].data(), M.lenm[1], n2, A + i, NMX, y.data(), 1);
        for (int j = 0; j < M.lenm[1]; ++j) A[j * NMX + i] = y[j];
      }
    }
  }
}
// map_to_face_space (mortar_operations.f90:353-447): restriction mortar -> face
template <class T> void map_to_face(const Mortar<T> &M, int side, const std::vector<T> &src, std::vector<T> &dst) {
  dst = src;
  if (M.conf[0][side] && M.conf[1][side]) return;
  int idir, jdir;
  side_dirs(M.orient, side, idir, jdir);
  const int n1 = M.len[idir][side], n2 = M.len[jdir][side];
  std::vector<T> t(NMX * NMX, T(0.0)), y(NMX);
  for (int v = 0; v < NV; ++v) {
    T *A = &dst[v * NMX * NMX];
    if (!M.conf[0][side]) {
      for (int j = 0; j < M.lenm[1]; ++j) apply1(M.Rm[side][0].data(), n1, M.lenm[0], A + j * NMX, 1, &t[j * NMX], 1);
      for (int j = 0; j < M.lenm[1]; ++j)
        for (int i = 0; i < n1; ++i) A[j * NMX + i] = t[j * NMX + i];
    }
    const int m1 = M.conf[0][side] ? M.lenm[0] : n1;
    if (!M.conf[1][side]) {
      for (int i = 0; i < m1; ++i) {
        apply1(M.Rm[side][1].data(), n2, M.lenm[1], A + i, NMX, y.data(), 1);
        for (int j = 0; j < n2; ++j) A[j * NMX + i] = y[j];
      }
    }
  }
}

// ------------------------------------------ boundary mortars (NS/BCs/stac3m)
// The external state of a wall: equal density and energy, normal momentum
// reversed (wallbc_Inv, wallbc_inv.f90:32-50; wallbc_isoth, wallbc_isoth2.f90:31-54).
template <class T> void wall_mirror(const double *nh, const T *Q1, T *Q2) {
  T qnorm = nh[0] * Q1[1] + nh[1] * Q1[2] + nh[2] * Q1[3];
  T q_tanx = Q1[1] - qnorm * nh[0];
  T q_tany = Q1[2] - qnorm * nh[1];
  T q_tanz = Q1[3] - qnorm * nh[2];
  Q2[0] = Q1[0];
  Q2[1] = q_tanx - qnorm * nh[0];
  Q2[2] = q_tany - qnorm * nh[1];
  Q2[3] = q_tanz - qnorm * nh[2];
  Q2[4] = Q1[4];
}

// osher (PhysLib.f90:698-790): the state between the two normal Riemann
// invariants and its Euler flux (fflux/gflux/hflux, PhysLib.f90:17-124).
template <class T> void osher(const double *nh, double ds, const T *Ql, const T *Qr, double gamma, T *flux) {
  const double en1 = nh[0], en2 = nh[1], en3 = nh[2];
  T rho = Ql[0], rhou = Ql[1], rhov = Ql[2], rhow = Ql[3], rhoe = Ql[4];
  T rhon = Qr[0], rhoun = Qr[1], rhovn = Qr[2], rhown = Qr[3], rhoen = Qr[4];
  T qdotn = (en1 * rhou + en2 * rhov + en3 * rhow) / rho;
  T qdotnn = (en1 * rhoun + en2 * rhovn + en3 * rhown) / rhon;
  T p = (gamma - 1.0) * (rhoe - 0.5 / rho * (rhou * rhou + rhov * rhov + rhow * rhow));
  T a = std::sqrt(gamma * p / rho);
  T pn = (gamma - 1.0) * (rhoen - 0.5 / rhon * (rhoun * rhoun + rhovn * rhovn + rhown * rhown));
  T an = std::sqrt(gamma * pn / rhon);
  T q_tanx = rhoun / rhon - qdotnn * en1;
  T q_tany = rhovn / rhon - qdotnn * en2;
  T q_tanz = rhown / rhon - qdotnn * en3;
  const double z = (gamma - 1.0) / (2.0 * gamma);
  T Ha = -qdotnn / an + 2.0 / (gamma - 1.0);
  Ha = Ha / (qdotn / a + 2.0 / (gamma - 1.0));
  pn = p / std::pow(Ha, 1.0 / z);
  T pstar = a + an - (qdotnn - qdotn) * (gamma - 1.0) / 2.0;
  pstar = pstar / (a / std::pow(p, z) + an / std::pow(pn, z));
  pstar = std::pow(pstar, 1.0 / z);
  T ustar = Ha * qdotn / a + qdotnn / an + 2.0 * (Ha - 1.0) / (gamma - 1.0);
  ustar = ustar / (Ha / a + 1.0 / an);
  T rho23 = pstar * gamma / (an * an);
  rho = rho23;
  p = pstar;
  qdotn = ustar;
  T u = q_tanx + en1 * qdotn, v = q_tany + en2 * qdotn, w = q_tanz + en3 * qdotn;
  T Q[NV] = {rho, rho * u, rho * v, rho * w, p / (gamma - 1.0) + 0.5 * rho * (u * u + v * v + w * w)};
  T f[NV], g[NV], h[NV];
  euler_fluxes(Q, gamma, f, g, h);
  for (int k = 0; k < NV; ++k) flux[k] = ds * (en1 * f[k] + en2 * g[k] + en3 * h[k]);
}

// riemann_solution (PhysLib.f90:326-412): the interface state from the normal
// Riemann invariants (used for the Dirichlet values of inflow and outflow).
template <class T> void riemann_solution(const double *nh, const T *Ql, const T *Qr, double gamma, T *Q) {
  const double en1 = nh[0], en2 = nh[1], en3 = nh[2];
  T rho = Ql[0], rhou = Ql[1], rhov = Ql[2], rhow = Ql[3], rhoe = Ql[4];
  T rhon = Qr[0], rhoun = Qr[1], rhovn = Qr[2], rhown = Qr[3], rhoen = Qr[4];
  T qdotn = (en1 * rhou + en2 * rhov + en3 * rhow) / rho;
  T qdotnn = (en1 * rhoun + en2 * rhovn + en3 * rhown) / rhon;
  T p = (gamma - 1.0) * (rhoe - 0.5 / rho * (rhou * rhou + rhov * rhov + rhow * rhow));
  T a = std::sqrt(gamma * p / rho);
  T pn = (gamma - 1.0) * (rhoen - 0.5 / rhon * (rhoun * rhoun + rhovn * rhovn + rhown * rhown));
  T an = std::sqrt(gamma * pn / rhon);
  T e0 = 0.5 * (qdotn + qdotnn);
  T eplus = e0 + 0.5 * (a + an);
  T eminus = e0 - 0.5 * (a + an);
  T etos, q_tanx, q_tany, q_tanz;
  if (re_(e0) > 0.0) {
    etos = p / std::pow(rho, gamma);
    q_tanx = rhou / rho - qdotn * en1;
    q_tany = rhov / rho - qdotn * en2;
    q_tanz = rhow / rho - qdotn * en3;
  } else {
    etos = pn / std::pow(rhon, gamma);
    q_tanx = rhoun / rhon - qdotnn * en1;
    q_tany = rhovn / rhon - qdotnn * en2;
    q_tanz = rhown / rhon - qdotnn * en3;
  }
  T rplus = re_(eplus) >= 0.0 ? qdotn + 2.0 / (gamma - 1.0) * a : qdotnn + 2.0 / (gamma - 1.0) * an;
  T rminus = re_(eminus) >= 0.0 ? qdotn - 2.0 / (gamma - 1.0) * a : qdotnn - 2.0 / (gamma - 1.0) * an;
  qdotn = 0.5 * (rplus + rminus);
  a = 0.25 * (gamma - 1.0) * (rplus - rminus);
  rho = std::pow(a * a / (gamma * etos), 1.0 / (gamma - 1.0));
  p = std::pow(rho, gamma) * etos;
  T u = q_tanx + en1 * qdotn, v = q_tany + en2 * qdotn, w = q_tanz + en3 * qdotn;
  Q[0] = rho;
  Q[1] = rho * u;
  Q[2] = rho * v;
  Q[3] = rho * w;
  Q[4] = p / (gamma - 1.0) + 0.5 * rho * (u * u + v * v + w * w);
}

// Inviscid boundary mortar: boundary_flux, then DirichletBC and send_q_to_faces
// (fluxesH_newa.f90:116-139; BackstepProblem-stoch.f90:1602-1689;
// wallbc_inv.f90, wallbc_isoth2.f90, inflow_specAll.f90, outflow_specAll.f90,
// set_adiabatic_wall / set_isothermal_wall / boundary_values in ViscousBC_slide.f90).
// Boundary mortars are conforming with orient 0: the master face only.
template <class T> void boundary_inviscid(Case<T> &c, Mortar<T> &M) {
  std::vector<T> Q1;
  gather_face(c, M, 0, c.el[M.id[0]].QL, Q1);
  Elem<T> &Em = c.el[M.id[0]];
  const bool low = (M.iface[0] == 1 || M.iface[0] == 3 || M.iface[0] == 6);
  const double cv = c.mach * c.mach * c.gamma * (c.gamma - 1.0);
  for (int j = 0; j < M.lenm[1]; ++j)
    for (int i = 0; i < M.lenm[0]; ++i) {
      const int pt = j * NMX + i;
      const double *nh = &M.n_hat[pt * 3];
      const double ds = M.norm[pt];
      T q1[NV], q2[NV], f[NV], qb[NV];
      for (int v = 0; v < NV; ++v) q1[v] = Q1[v * NMX * NMX + pt];
      if (M.bc == BC_WALLADIAB || M.bc == BC_WALLISOTH) {
        wall_mirror(nh, q1, q2);
        if (M.bc == BC_WALLADIAB) {
          riemann(nh, ds, low ? q2 : q1, low ? q1 : q2, c.gamma, f);
          qb[4] = q1[4];
        } else {
          T rho = q2[0], u = q2[1] / rho, v = q2[2] / rho, w = q2[3] / rho;
          q2[4] = rho * c.twall / cv + 0.5 * rho * (u * u + v * v + w * w);
          if (low) {
            const double mn[3] = {-nh[0], -nh[1], -nh[2]};
            osher(mn, -ds, q1, q2, c.gamma, f);
          } else {
            osher(nh, ds, q1, q2, c.gamma, f);
          }
          qb[4] = q1[0] * c.twall / cv;
        }
        qb[0] = q1[0];
        qb[1] = qb[2] = qb[3] = T(0.0);
      } else {  // inflow, outflow: the external state is the neighbour
        for (int v = 0; v < NV; ++v) q2[v] = T(M.Qx[v * NMX * NMX + pt]);
        riemann(nh, ds, low ? q2 : q1, low ? q1 : q2, c.gamma, f);
        riemann_solution(nh, low ? q2 : q1, low ? q1 : q2, c.gamma, qb);
      }
      for (int v = 0; v < NV; ++v) {
        face_ref(Em.F, Em, M.iface[0], i, j, v) = f[v];
        face_ref(Em.QL, Em, M.iface[0], i, j, v) = qb[v];
      }
    }
}

// Viscous boundary mortar: Vis_Neumann (BackstepProblem-stoch.f90:1693-1729)
// with wall_vis_flux / boundary_vis_flux (ViscousBC_slide.f90:183-348), then
// send_flux_to_faces_add on the master face.
template <class T> void boundary_viscous(Case<T> &c, Mortar<T> &M) {
  std::vector<T> r1;
  gather_face(c, M, 0, c.el[M.id[0]].R, r1);
  Elem<T> &Em = c.el[M.id[0]];
  for (int j = 0; j < M.lenm[1]; ++j)
    for (int i = 0; i < M.lenm[0]; ++i) {
      const int pt = j * NMX + i;
      const double nrm = M.norm[pt];
      for (int v = 0; v < NV; ++v) {
        T fv1 = r1[v * NMX * NMX + pt] / nrm;
        T qb;
        if (M.bc == BC_WALLADIAB || M.bc == BC_WALLISOTH) {
          qb = (v == 4 && M.bc == BC_WALLADIAB) ? T(0.0) : fv1 * nrm;
        } else {
          T Qs = T(M.fvx[v * NMX * NMX + pt]);
          if (M.nsign == -1) Qs = -Qs;
          qb = 0.5 * (fv1 + Qs) * nrm;
        }
        T &F = face_ref(Em.F, Em, M.iface[0], i, j, v);
        F = F - qb / c.re;
      }
    }
}

// Inviscid mortar: interface_flux + send_flux_to_faces + V_Avg_Soln + send_q_to_faces
// (mortar_operations.f90:151-238, 781-837; send_flux.f90:22-236; send_q.f90:21-280).
// Nonconforming faces use the consistent prolong -> flux/average -> restrict
// sequence (DSEM maps the averaged state twice and writes mortar-space data
// into face slots; those are documented deviations).
template <class T> void mortar_inviscid(Case<T> &c, Mortar<T> &M) {
  if (M.id[1] < 0) return boundary_inviscid(c, M);
  std::vector<T> Q1, Q2;
  gather_face(c, M, 0, c.el[M.id[0]].QL, Q1);
  gather_face(c, M, 1, c.el[M.id[1]].QL, Q2);
  rotate_to_mortar(M, Q2);
  map_to_mortar(M, 0, Q1);
  map_to_mortar(M, 1, Q2);
  std::vector<T> flux(NV * NMX * NMX, T(0.0)), avg(NV * NMX * NMX, T(0.0));
  const bool low = (M.iface[0] == 1 || M.iface[0] == 3 || M.iface[0] == 6);
  for (int j = 0; j < M.lenm[1]; ++j)
    for (int i = 0; i < M.lenm[0]; ++i) {
      T Ql[NV], Qr[NV], f[NV];
      for (int v = 0; v < NV; ++v) {
        T a = Q1[v * NMX * NMX + j * NMX + i], b = Q2[v * NMX * NMX + j * NMX + i];
        Ql[v] = low ? b : a;
        Qr[v] = low ? a : b;
      }
      riemann(&M.n_hat[(j * NMX + i) * 3], M.norm[j * NMX + i], Ql, Qr, c.gamma, f);
      for (int v = 0; v < NV; ++v) {
        flux[v * NMX * NMX + j * NMX + i] = f[v];
        T Qm = Q1[v * NMX * NMX + j * NMX + i], Qs = Q2[v * NMX * NMX + j * NMX + i];
        avg[v * NMX * NMX + j * NMX + i] = (Qm + Qs) * 0.5;
      }
    }
  // master side
  Elem<T> &Em = c.el[M.id[0]];
  std::vector<T> tf, tq;
  map_to_face(M, 0, flux, tf);
  map_to_face(M, 0, avg, tq);
  for (int v = 0; v < NV; ++v)
    for (int j = 0; j < M.len[1][0]; ++j)
      for (int i = 0; i < M.len[0][0]; ++i) {
        face_ref(Em.F, Em, M.iface[0], i, j, v) = tf[v * NMX * NMX + j * NMX + i];
        face_ref(Em.QL, Em, M.iface[0], i, j, v) = tq[v * NMX * NMX + j * NMX + i];
      }
  // slave side
  Elem<T> &Es = c.el[M.id[1]];
  map_to_face(M, 1, flux, tf);
  map_to_face(M, 1, avg, tq);
  rotate_to_face(M, tf);
  rotate_to_face(M, tq);
  const double sgn = (double)M.sign;
  for (int v = 0; v < NV; ++v)
    for (int j = 0; j < M.len[1][1]; ++j)
      for (int i = 0; i < M.len[0][1]; ++i) {
        face_ref(Es.F, Es, M.iface[1], i, j, v) = sgn * tf[v * NMX * NMX + j * NMX + i];
        face_ref(Es.QL, Es, M.iface[1], i, j, v) = tq[v * NMX * NMX + j * NMX + i];
      }
}

// Gauss_Deriv (SolnDerivsc.f90:14-83) of nf fields given on the three
// Lobatto grids: out[f][c][Gauss pt], c = x,y,z.
template <class T>
void gauss_deriv(const Elem<T> &E, const Ops &o, const T *const *w3, int nf, std::vector<T> &out) {
  const int G = E.G, L = E.L;
  const size_t ng = E.ng(), nl = E.nl();
  const int eg[3] = {G, G, G};
  std::vector<T> wd[3];
  for (int d = 0; d < 3; ++d) wd[d].resize(ng);
  out.assign((size_t)nf * 3 * ng, T(0.0));
  for (int f = 0; f < nf; ++f) {
    for (int d = 0; d < 3; ++d) {
      int el[3];
      grid_ext(d, G, L, el);
      contract(d, o.dmx.data(), G, L, w3[d] + f * nl, el, wd[d].data(), eg);
    }
    for (size_t p = 0; p < ng; ++p) {
      const double *gg = &E.gmetg[p * 9];
      for (int cc = 0; cc < 3; ++cc)
        out[((size_t)f * 3 + cc) * ng + p] = gg[0 + 3 * cc] * wd[0][p] + gg[1 + 3 * cc] * wd[1][p] + gg[2 + 3 * cc] * wd[2][p];
    }
  }
}

// Vis_Fluxes, element part (Vis_Fluxes_new.f90:57-231)
template <class T> void vis_element(Case<T> &c, Elem<T> &E) {
  const Ops &o = ops_for(E.G);
  const int G = E.G, L = E.L;
  const size_t ng = E.ng(), nl = E.nl();
  const T *w3[3] = {E.QL[0].data(), E.QL[1].data(), E.QL[2].data()};
  std::vector<T> gr;
  gauss_deriv(E, o, w3, NV, gr);
  const int eg[3] = {G, G, G};
  std::vector<T> gi(15 * nl);
  for (int d = 0; d < 3; ++d) {
    int el[3];
    grid_ext(d, G, L, el);
    for (int f = 0; f < 15; ++f) contract(d, o.bx.data(), L, G, &gr[f * ng], eg, &gi[f * nl], el);
    E.R[d].assign(NV * nl, T(0.0));
    for (int l = 0; l < el[2]; ++l)
      for (int m = 0; m < el[1]; ++m)
        for (int n = 0; n < el[0]; ++n) {
          size_t p = lidx(d, G, L, n, m, l);
          T Qv[NV], Qx[NV], Qy[NV], Qz[NV], f[NV], g[NV], h[NV];
          for (int v = 0; v < NV; ++v) {
            Qv[v] = E.QL[d][v * nl + p];
            Qx[v] = gi[(v * 3 + 0) * nl + p];
            Qy[v] = gi[(v * 3 + 1) * nl + p];
            Qz[v] = gi[(v * 3 + 2) * nl + p];
          }
          T amu = T(1.0);  // Vis_Fluxes_new.f90:123-125
          if (c.les) amu = amu + E.nut[d][p] * Qv[0];
          if (c.shock) amu = amu + E.muh[d][p];
          vis_fluxes(Qv, Qx, Qy, Qz, amu, c.gamma, c.pr, c.mach, f, g, h);
          const double *gm = &E.gmet[d][p * 3];
          int idx3[3] = {n, m, l};
          bool face = (idx3[d] == 0 || idx3[d] == L - 1);
          for (int v = 0; v < NV; ++v) {
            T r = gm[0] * f[v] + gm[1] * g[v] + gm[2] * h[v];
            E.R[d][v * nl + p] = r;
            if (!face) E.F[d][v * nl + p] = E.F[d][v * nl + p] - r / c.re;
          }
        }
  }
}

// Viscous mortar: send_flux_to_mortars (send_flux.f90:243-457),
// mortar_vis_flux (ViscousBC_slide.f90:231-271), send_flux_to_faces_add
// (send_flux.f90:699-921).  Conforming faces follow DSEM literally (the
// slave's fv is divided by the mortar norm at the slave's face index before
// rotation); nonconforming faces use the consistent prolong/restrict path.
template <class T> void mortar_viscous(Case<T> &c, Mortar<T> &M) {
  if (M.id[1] < 0) return boundary_viscous(c, M);
  std::vector<T> r1, r2;
  gather_face(c, M, 0, c.el[M.id[0]].R, r1);
  gather_face(c, M, 1, c.el[M.id[1]].R, r2);
  const bool conf1 = M.conf[0][0] && M.conf[1][0];
  const bool conf2 = M.conf[0][1] && M.conf[1][1];
  std::vector<T> fv1(NV * NMX * NMX, T(0.0)), fv2(NV * NMX * NMX, T(0.0));
  if (conf1) {
    for (int v = 0; v < NV; ++v)
      for (int j = 0; j < M.len[1][0]; ++j)
        for (int i = 0; i < M.len[0][0]; ++i)
          fv1[v * NMX * NMX + j * NMX + i] = r1[v * NMX * NMX + j * NMX + i] / M.norm[j * NMX + i];
  } else {
    map_to_mortar(M, 0, r1);
    for (int v = 0; v < NV; ++v)
      for (int j = 0; j < M.lenm[1]; ++j)
        for (int i = 0; i < M.lenm[0]; ++i)
          fv1[v * NMX * NMX + j * NMX + i] = r1[v * NMX * NMX + j * NMX + i] / M.norm[j * NMX + i];
  }
  if (conf2) {
    for (int v = 0; v < NV; ++v)
      for (int j = 0; j < M.len[1][1]; ++j)
        for (int i = 0; i < M.len[0][1]; ++i)
          fv2[v * NMX * NMX + j * NMX + i] = r2[v * NMX * NMX + j * NMX + i] / M.norm[j * NMX + i];
    rotate_to_mortar(M, fv2);
  } else {
    rotate_to_mortar(M, r2);
    map_to_mortar(M, 1, r2);
    for (int v = 0; v < NV; ++v)
      for (int j = 0; j < M.lenm[1]; ++j)
        for (int i = 0; i < M.lenm[0]; ++i)
          fv2[v * NMX * NMX + j * NMX + i] = r2[v * NMX * NMX + j * NMX + i] / M.norm[j * NMX + i];
  }
  std::vector<T> qb(NV * NMX * NMX, T(0.0));
  for (int j = 0; j < M.lenm[1]; ++j)
    for (int i = 0; i < M.lenm[0]; ++i)
      for (int v = 0; v < NV; ++v) {
        T Qs = fv2[v * NMX * NMX + j * NMX + i];
        if (M.nsign == -1) Qs = -Qs;
        T Qm = fv1[v * NMX * NMX + j * NMX + i];
        qb[v * NMX * NMX + j * NMX + i] = 0.5 * (Qm + Qs) * M.norm[j * NMX + i];
      }
  Elem<T> &Em = c.el[M.id[0]];
  std::vector<T> t;
  map_to_face(M, 0, qb, t);
  for (int v = 0; v < NV; ++v)
    for (int j = 0; j < M.len[1][0]; ++j)
      for (int i = 0; i < M.len[0][0]; ++i) {
        T &F = face_ref(Em.F, Em, M.iface[0], i, j, v);
        F = F - t[v * NMX * NMX + j * NMX + i] / c.re;
      }
  Elem<T> &Es = c.el[M.id[1]];
  std::vector<T> sq = qb;
  if (M.sign == -1)
    for (auto &x : sq) x = -x;
  map_to_face(M, 1, sq, t);
  rotate_to_face(M, t);
  for (int v = 0; v < NV; ++v)
    for (int j = 0; j < M.len[1][1]; ++j)
      for (int i = 0; i < M.len[0][1]; ++i) {
        T &F = face_ref(Es.F, Es, M.iface[1], i, j, v);
        F = F - t[v * NMX * NMX + j * NMX + i] / c.re;
      }
}

// Qt of one element (update_interior, updatea.f90:100-113, divergence part)
template <class T> void element_qt(const Elem<T> &E, std::vector<T> &Qt) {
  const Ops &o = ops_for(E.G);
  const int G = E.G, L = E.L;
  const size_t ng = E.ng(), nl = E.nl();
  const int eg[3] = {G, G, G};
  Qt.assign(NV * ng, T(0.0));
  std::vector<T> S[3];
  for (int d = 0; d < 3; ++d) S[d].resize(ng);
  for (int v = 0; v < NV; ++v) {
    for (int d = 0; d < 3; ++d) {
      int el[3];
      grid_ext(d, G, L, el);
      contract(d, o.dmx.data(), G, L, &E.F[d][v * nl], el, S[d].data(), eg, 1, L - 1);
    }
    for (int l = 0; l < G; ++l)
      for (int m = 0; m < G; ++m)
        for (int n = 0; n < G; ++n) {
          size_t p = gidx(G, n, m, l);
          const T *F0 = &E.F[0][v * nl], *F1 = &E.F[1][v * nl], *F2 = &E.F[2][v * nl];
          T acc = S[2][p] + S[1][p] + S[0][p];  // z, y, x: the CUDA kernel's pass order
          acc = fmac(o.dmx[n * L + 0], F0[lidx(0, G, L, 0, m, l)], acc);
          acc = fmac(o.dmx[n * L + L - 1], F0[lidx(0, G, L, L - 1, m, l)], acc);
          acc = fmac(o.dmx[m * L + 0], F1[lidx(1, G, L, n, 0, l)], acc);
          acc = fmac(o.dmx[m * L + L - 1], F1[lidx(1, G, L, n, L - 1, l)], acc);
          acc = fmac(o.dmx[l * L + 0], F2[lidx(2, G, L, n, m, 0)], acc);
          acc = fmac(o.dmx[l * L + L - 1], F2[lidx(2, G, L, n, m, L - 1)], acc);
          Qt[v * ng + p] = -acc;
        }
  }
}

// Fluxes (fluxesH_newa.f90:17-199)
template <class T> void fluxes(Case<T> &c) {
  const int ne = (int)c.el.size(), nm = (int)c.mo.size();
#pragma omp parallel for schedule(dynamic, 4)
  for (int e = 0; e < ne; ++e) int_fluxes(c, c.el[e]);
#pragma omp parallel for schedule(dynamic, 16)
  for (int j = 0; j < nm; ++j) mortar_inviscid(c, c.mo[j]);
#pragma omp parallel for schedule(dynamic, 4)
  for (int e = 0; e < ne; ++e) vis_element(c, c.el[e]);
#pragma omp parallel for schedule(dynamic, 16)
  for (int j = 0; j < nm; ++j) mortar_viscous(c, c.mo[j]);
  c.ql_valid = true;
}

// ---------------------------------------- entropy viscosity (EV_routines)
// calculate_terms (RHS.f90:207-278): only RHS (and the Ducros sensor) feed the viscosity.
template <class T>
T ev_residual(const Case<T> &c, const T *Q, const T *Qx, const T *Qy, const T *Qz, const T *T1, T &ducros) {
  const double gamma = c.gamma;
  T rho = Q[0], rhou = Q[1], rhov = Q[2], rhow = Q[3], rhoe = Q[4];
  T u = rhou / rho, v = rhov / rho, w = rhow / rho;
  T p = (gamma - 1.0) * (rhoe - 0.5 * rho * (u * u + v * v + w * w));
  T Tt = p * gamma / rho;
  T ux = (Qx[1] - u * Qx[0]) / rho, uy = (Qy[1] - u * Qy[0]) / rho, uz = (Qz[1] - u * Qz[0]) / rho;
  T vx = (Qx[2] - v * Qx[0]) / rho, vy = (Qy[2] - v * Qy[0]) / rho, vz = (Qz[2] - v * Qz[0]) / rho;
  T wx = (Qx[3] - w * Qx[0]) / rho, wy = (Qy[3] - w * Qy[0]) / rho, wz = (Qz[3] - w * Qz[0]) / rho;
  T tx = T1[0], ty = T1[1], tz = T1[2];
  T phi = (2.0 * (ux * ux + vy * vy + wz * wz) +
           ((vx + uy) * (vx + uy) + (uz + wx) * (uz + wx) + (vz + wy) * (vz + wy)) -
           2.0 * ((ux + vy + wz) * (ux + vy + wz)) / 3.0);
  T gam = (tx * tx + ty * ty + tz * tz) / (Tt * (gamma - 1.0) * c.pr);
  T div = ux + vy + wz;
  T cur = std::sqrt((wy - vz) * (wy - vz) + (uz - wx) * (uz - wx) + (vx - uy) * (vx - uy));
  ducros = rmax(T(0.0), rmin(T(1.0), (div * div / (div * div + cur * cur + 1.0e-9))));
  return (((phi + gam) / Tt) / c.re);
}

// Density-based sensor of calculate_terms (RHS.f90:264-275) from the density gradient.
template <class T> T rho_sensor(const T &rx, const T &ry, const T &rz) {
  const double eps = 1.0e-9;
  T rhoX2 = rx * rx, rhoY2 = ry * ry, rhoZ2 = rz * rz;
  return std::sqrt((1.0 / ((1.0 / (rhoX2 + eps)) + (1.0 / (rhoY2 + eps)) + 1.0)) +
                   (1.0 / ((1.0 / (rhoX2 + eps)) + (1.0 / (rhoZ2 + eps)) + 1.0)) +
                   (1.0 / ((1.0 / (rhoY2 + eps)) + (1.0 / (rhoZ2 + eps)) + 1.0)));
}

// Entropy (EV_routines/Main/Driver.f90:21-60): RHS_ent_trans (RHS.f90:21-190),
// Entropy_Viscosity (EViscosity_GL.f90:19-101), EV_Prolong (Prolong_gtol.f90:7-51).
// Uses the Lobatto arrays left by the previous Fluxes call; before any Fluxes
// call (and wherever the coefficient is not finite) the viscosity is 0.
template <class T> void entropy(Case<T> &c) {
  const int ne = (int)c.el.size();
#pragma omp parallel for schedule(dynamic, 4)
  for (int e = 0; e < ne; ++e) {
    Elem<T> &E = c.el[e];
    const Ops &o = ops_for(E.G);
    const int G = E.G, L = E.L;
    const size_t ng = E.ng(), nl = E.nl();
    E.muhg.assign(ng, T(0.0));
    if (c.ql_valid) {
      std::vector<T> Tl[3];
      for (int d = 0; d < 3; ++d) {
        Tl[d].resize(nl);
        const T *q = E.QL[d].data();
        for (size_t p = 0; p < nl; ++p) {
          T q1 = q[p], q2 = q[nl + p], q3 = q[2 * nl + p], q4 = q[3 * nl + p], q5 = q[4 * nl + p];
          T P = (c.gamma - 1.0) * (q5 - 0.5 * q1 * ((q2 / q1) * (q2 / q1) + (q3 / q1) * (q3 / q1) + (q4 / q1) * (q4 / q1)));
          Tl[d][p] = P * c.gamma / q1;
        }
      }
      const T *w3[3] = {E.QL[0].data(), E.QL[1].data(), E.QL[2].data()};
      const T *t3[3] = {Tl[0].data(), Tl[1].data(), Tl[2].data()};
      std::vector<T> gq, gt;
      gauss_deriv(E, o, w3, 4, gq);
      gauss_deriv(E, o, t3, 1, gt);
      for (size_t p = 0; p < ng; ++p) {
        T Q[NV], Qx[NV], Qy[NV], Qz[NV], T1[3];
        for (int v = 0; v < NV; ++v) Q[v] = E.Q[v * ng + p] * E.jacob[p];
        for (int v = 0; v < 4; ++v) {
          Qx[v] = gq[(v * 3 + 0) * ng + p];
          Qy[v] = gq[(v * 3 + 1) * ng + p];
          Qz[v] = gq[(v * 3 + 2) * ng + p];
        }
        Qx[4] = Qy[4] = Qz[4] = T(0.0);
        for (int k = 0; k < 3; ++k) T1[k] = gt[k * ng + p];
        T duc;
        T biS = ev_residual(c, Q, Qx, Qy, Qz, T1, duc);
        E.ducros[p] = duc;  // the sensors the Smagorinsky model reads (RHS.f90:180-181)
        E.rhos[p] = rho_sensor(Qx[0], Qy[0], Qz[0]);
        T rho = E.Q[p] * E.jacob[p];
        double h = E.hdelta[p];
        T mur = c.cmu * c.re * rho * (h * h) * rabs(biS);
        if (c.ducros) mur = mur * duc;
        T mu = rmin(rmax(mur, T(0.0)), T(c.mumax));
        if (!rfinite(mu)) mu = T(0.0);
        E.muhg[p] = mu;
      }
    }
    const int eg[3] = {G, G, G};
    for (int d = 0; d < 3; ++d) {
      int el[3];
      grid_ext(d, G, L, el);
      E.muh[d].resize(nl);
      contract(d, o.bx.data(), L, G, E.muhg.data(), eg, E.muh[d].data(), el);
    }
  }
}

// Static Smagorinsky viscosity (simpleSmag, turbulence/staticSmago/staticSmag.f90:32-118,
// filteredStrain :126-183, delta_g :191-201) from the last Fluxes call's Lobatto
// arrays, and nut_prolong (:206-261).  DSEM forms rho from jacob(1,1,1) of the
// element and the velocities from d%Q without the Jacobian; both kept.
template <class T> void smagorinsky(Case<T> &c) {
  const int ne = (int)c.el.size();
#pragma omp parallel for schedule(dynamic, 4)
  for (int e = 0; e < ne; ++e) {
    Elem<T> &E = c.el[e];
    const Ops &o = ops_for(E.G);
    const int G = E.G, L = E.L;
    const size_t ng = E.ng(), nl = E.nl();
    std::vector<T> gq((size_t)4 * 3 * ng, T(0.0));
    if (c.ql_valid) {
      const T *w3[3] = {E.QL[0].data(), E.QL[1].data(), E.QL[2].data()};
      gauss_deriv(E, o, w3, 4, gq);
    }
    E.nutg.assign(ng, T(0.0));
    for (size_t p = 0; p < ng; ++p) {
      auto Qx = [&](int v) { return gq[(v * 3 + 0) * ng + p]; };
      auto Qy = [&](int v) { return gq[(v * 3 + 1) * ng + p]; };
      auto Qz = [&](int v) { return gq[(v * 3 + 2) * ng + p]; };
      T rho = E.Q[p] * E.jacob[0];
      T u = E.Q[ng + p] / rho, v = E.Q[2 * ng + p] / rho, w = E.Q[3 * ng + p] / rho;
      T rho_x = Qx(0), rho_y = Qy(0), rho_z = Qz(0);
      T u_x = (Qx(1) - rho_x * u) / rho, u_y = (Qy(1) - rho_y * u) / rho, u_z = (Qz(1) - rho_z * u) / rho;
      T v_x = (Qx(2) - rho_x * v) / rho, v_y = (Qy(2) - rho_y * v) / rho, v_z = (Qz(2) - rho_z * v) / rho;
      T w_x = (Qx(3) - rho_x * w) / rho, w_y = (Qy(3) - rho_y * w) / rho, w_z = (Qz(3) - rho_z * w) / rho;
      T S11 = u_x, S12 = 0.5 * (u_y + v_x), S13 = 0.5 * (u_z + w_x);
      T S21 = 0.5 * (v_x + u_y), S22 = v_y, S23 = 0.5 * (v_z + w_y);
      T S31 = 0.5 * (w_x + u_z), S32 = 0.5 * (w_y + v_z), S33 = w_z;
      T S = std::sqrt(2.0 * S11 * S11 + 2.0 * S12 * S12 + 2.0 * S13 * S13 + 2.0 * S21 * S21 + 2.0 * S22 * S22 +
                      2.0 * S23 * S23 + 2.0 * S31 * S31 + 2.0 * S32 * S32 + 2.0 * S33 * S33);
      const double dg = E.hdelta[p];
      T nu = c.re * (c.cs * dg) * (c.cs * dg) * S;
      if (c.shock_sensor) nu = nu * (1.0 - E.ducros[p]);  // staticSmag.f90:68-69
      if (c.rho_sensor) nu = nu * E.rhos[p];
      E.nutg[p] = rmin(rmax(nu, T(0.0)), T(c.numax));
    }
    const int eg[3] = {G, G, G};
    for (int d = 0; d < 3; ++d) {
      int el[3];
      grid_ext(d, G, L, el);
      E.nut[d].resize(nl);
      contract(d, o.bx.data(), L, G, E.nutg.data(), eg, E.nut[d].data(), el);
      for (auto &x : E.nut[d])
        if (re_(x) < 0.0) x = T(0.0);
    }
  }
}

// ----------------------------------------------------------------- stage
template <class T> double update_all(Case<T> &c, double dt, int kk, double *Qt_out, int ldx) {
  const int ne = (int)c.el.size();
  double resid = 0.0;
  bool bad = false;
#pragma omp parallel for schedule(dynamic, 4) reduction(max : resid) reduction(|| : bad)
  for (int e = 0; e < ne; ++e) {
    Elem<T> &E = c.el[e];
    std::vector<T> Qt;
    element_qt(E, Qt);
    const size_t ng = E.ng();
    const int G = E.G;
    for (size_t i = 0; i < NV * ng; ++i) {
      double a = std::fabs(re_(Qt[i]));
      if (!(a == a) || std::isinf(a)) bad = true;
      resid = std::max(resid, a);
    }
    if (Qt_out) {
      for (int v = 0; v < NV; ++v)
        for (int l = 0; l < G; ++l)
          for (int m = 0; m < G; ++m)
            for (int n = 0; n < G; ++n)
              Qt_out[(size_t)e * NV * ldx * ldx * ldx + n + (size_t)ldx * (m + (size_t)ldx * (l + (size_t)ldx * v))] =
                  re_(Qt[v * ng + gidx(G, n, m, l)]);
    }
    if (kk > 0) {
      const double a = c.ark[kk - 1], cc = c.crk[kk - 1];
      for (size_t i = 0; i < NV * ng; ++i) {
        E.gQ[i] = a * E.gQ[i] + Qt[i];
        E.Q[i] = E.Q[i] + cc * dt * E.gQ[i];
      }
    }
  }
  return bad ? NAN : resid;
}

template <class T> int stage(Case<T> &c, double time, double dt, int kk, double *Qt, int ldx) {
  if (kk == 1) {
    if (c.shock) entropy(c);
    if (c.les) smagorinsky(c);
    for (auto &E : c.el) std::fill(E.gQ.begin(), E.gQ.end(), T(0.0));
  }
  (void)time;
  fluxes(c);
  double r = update_all(c, dt, kk, Qt, ldx);
  return std::isfinite(r) ? 0 : -3;
}

// ------------------------------------------------------------- mesh build
// Face_Map_hex8 (element_library.f90), faces 1..6 -> local corner numbers
const int face_map[6][4] = {{0, 1, 5, 4}, {3, 2, 6, 7}, {0, 1, 2, 3}, {1, 2, 6, 5}, {4, 5, 6, 7}, {0, 3, 7, 4}};
const int edge_map[6][2] = {{0, 2}, {0, 2}, {0, 1}, {1, 2}, {0, 1}, {1, 2}};
// sign_map (set_mortars.f90:113-118), [ifl][ifr]
const int sign_map[6][6] = {{-1, 1, -1, 1, 1, -1}, {1, -1, 1, -1, -1, 1}, {-1, 1, -1, 1, 1, -1},
                            {1, -1, 1, -1, -1, 1},  {1, -1, 1, -1, -1, 1}, {-1, 1, -1, 1, 1, -1}};
// faces_match orientation (face_operations.f90:404-456, element_library.f90:99-146)
int side_map(int a, int b) {  // 0-based corners of a face
  static const int sm[4][4] = {{-99, 1, -99, 2}, {-1, -99, 2, -99}, {-99, -2, -99, -1}, {-2, -99, 1, -99}};
  return sm[a][b];
}
int orient_map(int is1, int is2) {
  if (is1 == 1 && is2 == 2) return 0;
  if (is1 == -1 && is2 == 2) return 1;
  if (is1 == -1 && is2 == -2) return 2;
  if (is1 == 1 && is2 == -2) return 3;
  if (is1 == 2 && is2 == 1) return 4;
  if (is1 == -2 && is2 == 1) return 5;
  if (is1 == -2 && is2 == -1) return 6;
  if (is1 == 2 && is2 == -1) return 7;
  return -99;
}
bool faces_match(const int *tn, const int *sn, int &orient) {
  int cc[4];
  for (int i = 0; i < 4; ++i) {
    bool hit = false;
    for (int k = 0; k < 4; ++k)
      if (tn[i] == sn[k]) {
        hit = true;
        cc[i] = k;
        break;
      }
    if (!hit) return false;
  }
  orient = orient_map(side_map(cc[0], cc[1]), side_map(cc[0], cc[3]));
  return true;
}

// 24 proper rotations of the reference cube: signed permutations, det +1.
void rotation_matrix(int r, int R[3][3]) {
  static int mats[24][3][3];
  static bool init = false;
  if (!init) {
    int cnt = 0;
    const int perms[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2}, {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
    for (int pi = 0; pi < 6; ++pi)
      for (int s = 0; s < 8; ++s) {
        int M[3][3] = {};
        for (int i = 0; i < 3; ++i) M[i][perms[pi][i]] = (s >> i & 1) ? -1 : 1;
        int det = M[0][0] * (M[1][1] * M[2][2] - M[1][2] * M[2][1]) - M[0][1] * (M[1][0] * M[2][2] - M[1][2] * M[2][0]) +
                  M[0][2] * (M[1][0] * M[2][1] - M[1][1] * M[2][0]);
        if (det != 1) continue;
        std::memcpy(mats[cnt++], M, sizeof(M));
      }
    init = true;
  }
  std::memcpy(R, mats[r % 24], sizeof(int) * 9);
}
const int corner_xyz[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0}, {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};

template <class T> void set_geometry(Elem<T> &E) {
  const Ops &o = ops_for(E.G);
  const int G = E.G, L = E.L;
  const size_t ng = E.ng(), nl = E.nl();
  E.jacob.resize(ng);
  E.gmetg.resize(9 * ng);
  E.xg.resize(3 * ng);
  E.hdelta.resize(ng);
  for (int l = 0; l < G; ++l)
    for (int m = 0; m < G; ++m)
      for (int n = 0; n < G; ++n) {
        double cx[3] = {o.cxg[n], o.cxg[m], o.cxg[l]}, gx[3][3], gc[3][3], J;
        size_t p = gidx(G, n, m, l);
        hex8_map(E.corner, cx, &E.xg[3 * p]);
        grad_hex8_map(E.corner, cx, gx);
        invert_metric(gx, gc, J);
        E.jacob[p] = 1.0 / J;
        for (int a = 0; a < 3; ++a)
          for (int b = 0; b < 3; ++b) E.gmetg[p * 9 + a + 3 * b] = gc[a][b];
      }
  for (int d = 0; d < 3; ++d) {
    E.gmet[d].resize(3 * nl);
    int el[3];
    grid_ext(d, G, L, el);
    for (int l = 0; l < el[2]; ++l)
      for (int m = 0; m < el[1]; ++m)
        for (int n = 0; n < el[0]; ++n) {
          double cx[3] = {d == 0 ? o.cx[n] : o.cxg[n], d == 1 ? o.cx[m] : o.cxg[m], d == 2 ? o.cx[l] : o.cxg[l]};
          double gx[3][3], gc[3][3], J;
          grad_hex8_map(E.corner, cx, gx);
          invert_metric(gx, gc, J);
          size_t p = lidx(d, G, L, n, m, l);
          for (int b = 0; b < 3; ++b) E.gmet[d][p * 3 + b] = J * gc[d][b];
        }
  }
  for (size_t p = 0; p < ng; ++p)  // delta_g (staticSmag.f90:191-201)
    E.hdelta[p] = std::pow(std::fabs(1.0 / E.jacob[p]), 1.0 / 3.0) / std::pow((double)(G * G * G), 1.0 / 3.0);
}

// mortar geometry from the master element (set_domain_geometry.f90:258-345)
template <class T> void mortar_geometry(Elem<T> &E, int face, Mortar<T> &M) {
  static const double end_vals[6] = {0.0, 1.0, 0.0, 1.0, 1.0, 0.0};
  std::vector<double> c1(M.lenm[0]), c2(M.lenm[1]);
  gauss_points(M.lenm[0], c1.data());
  gauss_points(M.lenm[1], c2.data());
  M.n_hat.assign(NMX * NMX * 3, 0.0);
  M.norm.assign(NMX * NMX, 0.0);
  const int d = (face == 1 || face == 2) ? 1 : (face == 3 || face == 5) ? 2 : 0;
  for (int j = 0; j < M.lenm[1]; ++j)
    for (int i = 0; i < M.lenm[0]; ++i) {
      double cx[3];
      if (d == 1) { cx[1] = end_vals[face - 1]; cx[0] = c1[i]; cx[2] = c2[j]; }
      else if (d == 2) { cx[2] = end_vals[face - 1]; cx[0] = c1[i]; cx[1] = c2[j]; }
      else { cx[0] = end_vals[face - 1]; cx[1] = c1[i]; cx[2] = c2[j]; }
      double gx[3][3], gc[3][3], J;
      grad_hex8_map(E.corner, cx, gx);
      invert_metric(gx, gc, J);
      double sqr = std::sqrt(gc[d][0] * gc[d][0] + gc[d][1] * gc[d][1] + gc[d][2] * gc[d][2]);
      for (int k = 0; k < 3; ++k) M.n_hat[(j * NMX + i) * 3 + k] = gc[d][k] / sqr;
      M.norm[j * NMX + i] = J * sqr;
    }
}

// set_mortar_nsign (set_mortars.f90:240-372), including the face-5 index quirk
template <class T> void face_normal(const Elem<T> &E, int face, double n[3]) {
  const int G = E.G, L = E.L;
  size_t p;
  int d;
  switch (face) {
    case 1: d = 1; p = lidx(1, G, L, 0, 0, 0); break;
    case 2: d = 1; p = lidx(1, G, L, 0, L - 1, 0); break;
    case 3: d = 2; p = lidx(2, G, L, 0, 0, 0); break;
    case 4: d = 0; p = lidx(0, G, L, L - 1, 0, 0); break;
    case 5: d = 2; p = lidx(2, G, L, 0, 0, L - 1); break;
    default: d = 0; p = lidx(0, G, L, 0, 0, 0); break;
  }
  const double *g = &E.gmet[d][p * 3];
  double sqr = std::sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
  n[0] = g[0] / sqr;
  n[1] = g[1] / sqr;
  n[2] = g[2] / sqr;
  // DSEM's face-5 branch reads the third component at gmet(3,3,1,nc,1), an
  // entry outside the z-grid's Gauss extent in y (set_mortars.f90:293-297);
  // the oracle uses the face's own metric, which is what that line intends.
}

template <class T> void set_mortar_matrices(Mortar<T> &M) {  // mortarLib.f90:27-186
  for (int side = 0; side < 2; ++side)
    for (int dir = 0; dir < 2; ++dir) {
      if (M.conf[dir][side]) continue;
      int idirt = dir;
      if (side == 1 && M.orient >= 4) idirt = 1 - dir;
      const int nin = M.len[idirt][side], nout = M.lenm[dir];
      std::vector<double> cin(nin), cout_(nout);
      gauss_points(nin, cin.data());
      gauss_points(nout, cout_.data());
      M.P[side][dir].resize(nout * nin);
      M.Rm[side][dir].resize(nin * nout);
      compute_pmat(cin.data(), nin, cout_.data(), nout, M.P[side][dir].data());
      compute_pmat(cout_.data(), nout, cin.data(), nin, M.Rm[side][dir].data());
      M.pin[side][dir] = nin;
    }
}

template <class T> void finish_mortar(Mortar<T> &M, const Case<T> &c) {
  const Elem<T> &Em = c.el[M.id[0]];
  const Elem<T> &Es = c.el[M.id[1]];
  const int ifl = M.iface[0], ifr = M.iface[1];
  M.len[0][0] = Em.G;  // isotropic orders: ncg along both face directions
  M.len[1][0] = Em.G;
  M.len[0][1] = Es.G;
  M.len[1][1] = Es.G;
  (void)ifl;
  (void)ifr;
  int j1 = 0, j2 = 1;
  if (M.orient >= 4) { j1 = 1; j2 = 0; }
  M.lenm[0] = std::max(M.len[0][0], M.len[j1][1]);
  M.lenm[1] = std::max(M.len[1][0], M.len[j2][1]);
  M.conf[0][0] = M.lenm[0] == M.len[0][0];
  M.conf[1][0] = M.lenm[1] == M.len[1][0];
  M.conf[0][1] = M.lenm[0] == M.len[j1][1];
  M.conf[1][1] = M.lenm[1] == M.len[j2][1];
}

template <class T> Case<T> *build_box(int nex, int ney, int nez, double lx, double ly, double lz, const int *orders,
                                      const int *rot) {
  auto *c = new Case<T>();
  rkcoefs(*c, 4);
  const int ne = nex * ney * nez;
  c->el.resize(ne);
  auto nid = [&](int ix, int iy, int iz) { return iy + (ney + 1) * (ix + (nex + 1) * iz); };
  for (int iz = 0; iz < nez; ++iz)
    for (int ix = 0; ix < nex; ++ix)
      for (int iy = 0; iy < ney; ++iy) {
        const int e = iy + ney * (ix + nex * iz);
        Elem<T> &E = c->el[e];
        E.G = orders[e] + 1;
        E.L = E.G + 1;
        int base[8], R[3][3];
        double bc[8][3];
        for (int k = 0; k < 8; ++k) {
          int a = ix + corner_xyz[k][0], b = iy + corner_xyz[k][1], cc = iz + corner_xyz[k][2];
          base[k] = nid(a, b, cc);
          bc[k][0] = a * (lx / nex);
          bc[k][1] = b * (ly / ney);
          bc[k][2] = cc * (lz / nez);
        }
        rotation_matrix(rot ? rot[e] : 0, R);
        for (int k = 0; k < 8; ++k) {  // new corner k sits at old local coords R^T(xi_k - .5) + .5
          int src[3];
          for (int a = 0; a < 3; ++a) {
            int s = 0;
            for (int b = 0; b < 3; ++b) s += R[b][a] * (2 * corner_xyz[k][b] - 1);
            src[a] = (s + 1) / 2;
          }
          int kk = 0;
          for (int q = 0; q < 8; ++q)
            if (corner_xyz[q][0] == src[0] && corner_xyz[q][1] == src[1] && corner_xyz[q][2] == src[2]) kk = q;
          E.node[k] = base[kk];
          for (int a = 0; a < 3; ++a) E.corner[k][a] = bc[kk][a];
        }
        const size_t ng = E.ng();
        E.Q.assign(NV * ng, T(0.0));
        E.gQ.assign(NV * ng, T(0.0));
    E.ducros.assign(ng, T(0.0));
    E.rhos.assign(ng, T(0.0));
      }
  // generate_mortars (set_mortars.f90:20-224): first element to present a face is the master
  std::map<std::array<int, 4>, int> faces;
  for (int e = 0; e < ne; ++e) {
    Elem<T> &E = c->el[e];
    for (int f = 0; f < 6; ++f) {
      int fn[4];
      for (int k = 0; k < 4; ++k) fn[k] = E.node[face_map[f][k]];
      std::array<int, 4> key = {fn[0], fn[1], fn[2], fn[3]};
      std::sort(key.begin(), key.end());
      auto it = faces.find(key);
      if (it == faces.end()) {
        Mortar<T> M;
        M.id[0] = e;
        M.iface[0] = f + 1;
        M.id[1] = -1;
        faces[key] = (int)c->mo.size();
        E.mort[f] = (int)c->mo.size();
        E.mside[f] = 1;
        E.boundary[f] = true;
        c->mo.push_back(M);
      } else {
        Mortar<T> &M = c->mo[it->second];
        Elem<T> &Em = c->el[M.id[0]];
        int mn[4];
        for (int k = 0; k < 4; ++k) mn[k] = Em.node[face_map[M.iface[0] - 1][k]];
        int orient = 0;
        faces_match(mn, fn, orient);
        M.id[1] = e;
        M.iface[1] = f + 1;
        M.orient = orient;
        M.sign = sign_map[M.iface[0] - 1][f];
        E.orientation[f] = orient;
        E.mort[f] = it->second;
        E.mside[f] = 2;
        Em.boundary[M.iface[0] - 1] = false;
      }
    }
  }
  for (auto &M : c->mo) {
    if (M.id[1] < 0) {
      const Elem<T> &Em = c->el[M.id[0]];
      M.len[0][0] = Em.G;
      M.len[1][0] = Em.G;
      M.lenm[0] = M.lenm[1] = Em.G;
    } else {
      finish_mortar(M, *c);
    }
  }
  for (auto &E : c->el) set_geometry(E);
  for (int e = 0; e < ne; ++e)
    for (int f = 0; f < 6; ++f)
      if (c->el[e].mside[f] == 1) mortar_geometry(c->el[e], f + 1, c->mo[c->el[e].mort[f]]);
  // user_setup periodic pairing (caseFiles/tgv/BackstepProblem-stoch.f90:173-278)
  std::vector<int> removed(c->mo.size(), 0);
  auto pair = [&](int idm, int fm, int ids, int fs, bool master_is_m) {
    Elem<T> &Em = c->el[idm];
    Elem<T> &Es = c->el[ids];
    int keep = master_is_m ? Em.mort[fm - 1] : Es.mort[fs - 1];
    int drop = master_is_m ? Es.mort[fs - 1] : Em.mort[fm - 1];
    Mortar<T> &M = c->mo[keep];
    int mel = master_is_m ? idm : ids, sel = master_is_m ? ids : idm;
    int mf = master_is_m ? fm : fs, sf = master_is_m ? fs : fm;
    M.id[0] = mel;
    M.iface[0] = mf;
    M.id[1] = sel;
    M.iface[1] = sf;
    M.len[0][1] = c->el[sel].G;
    M.len[1][1] = c->el[sel].G;
    removed[drop] = 1;
    c->el[sel].mort[sf - 1] = keep;
    c->el[sel].mside[sf - 1] = 2;
    Em.boundary[fm - 1] = false;
    Es.boundary[fs - 1] = false;
  };
  for (int idm = 0; idm < ne; ++idm)  // z: face 3 master, face 5 slave
    if (c->el[idm].boundary[2])
      for (int ids = 0; ids < ne; ++ids)
        if (c->el[ids].boundary[4] && c->el[idm].corner[0][0] == c->el[ids].corner[4][0] &&
            c->el[idm].corner[0][1] == c->el[ids].corner[4][1]) {
          pair(idm, 3, ids, 5, true);
          break;
        }
  for (int idm = 0; idm < ne; ++idm)  // y: face 1 master, face 2 slave
    if (c->el[idm].boundary[0])
      for (int ids = 0; ids < ne; ++ids)
        if (c->el[ids].boundary[1] && c->el[idm].corner[0][0] == c->el[ids].corner[3][0] &&
            c->el[idm].corner[0][2] == c->el[ids].corner[3][2]) {
          pair(idm, 1, ids, 2, true);
          break;
        }
  for (int idm = 0; idm < ne; ++idm)  // x: face 4 (of ids) master, face 6 slave
    if (c->el[idm].boundary[5])
      for (int ids = 0; ids < ne; ++ids)
        if (c->el[ids].boundary[3] && c->el[idm].corner[0][2] == c->el[ids].corner[1][2] &&
            c->el[idm].corner[0][1] == c->el[ids].corner[1][1]) {
          pair(idm, 6, ids, 4, false);
          break;
        }
  std::vector<Mortar<T>> kept;
  std::vector<int> newid(c->mo.size(), -1);
  for (size_t j = 0; j < c->mo.size(); ++j)
    if (!removed[j]) {
      newid[j] = (int)kept.size();
      kept.push_back(c->mo[j]);
    }
  c->mo.swap(kept);
  for (auto &E : c->el)
    for (int f = 0; f < 6; ++f) E.mort[f] = newid[E.mort[f]];
  for (auto &M : c->mo) {
    double n1[3], n2[3];
    face_normal(c->el[M.id[0]], M.iface[0], n1);
    face_normal(c->el[M.id[1]], M.iface[1], n2);
    double sj = n1[0] * n2[0] + n1[1] * n2[1] + n1[2] * n2[2];
    M.nsign = sj >= 0 ? 1 : -1;
    set_mortar_matrices(M);
  }
  return c;
}

template <class T> void export_desc(const Case<T> &c, int ldx, int *ncg, double *jacob, double *gmetg, double *gmet,
                                    int *mortar, double *n_hat, double *norm, double *xg) {
  const size_t L3 = (size_t)ldx * ldx * ldx;
  for (size_t e = 0; e < c.el.size(); ++e) {
    const Elem<T> &E = c.el[e];
    const int G = E.G, L = E.L;
    if (ncg) ncg[3 * e] = ncg[3 * e + 1] = ncg[3 * e + 2] = G;
    for (int l = 0; l < L; ++l)
      for (int m = 0; m < L; ++m)
        for (int n = 0; n < L; ++n) {
          size_t q = n + (size_t)ldx * (m + (size_t)ldx * l);
          if (n < G && m < G && l < G) {
            size_t p = gidx(G, n, m, l);
            if (jacob) jacob[e * L3 + q] = E.jacob[p];
            if (gmetg)
              for (int k = 0; k < 9; ++k) gmetg[(e * L3 + q) * 9 + k] = E.gmetg[p * 9 + k];
            if (xg)
              for (int k = 0; k < 3; ++k) xg[(e * L3 + q) * 3 + k] = E.xg[p * 3 + k];
          }
          if (gmet)
            for (int d = 0; d < 3; ++d) {
              int idx3[3] = {n, m, l};
              bool ok = true;
              for (int a = 0; a < 3; ++a)
                if (idx3[a] >= (a == d ? L : G)) ok = false;
              if (!ok) continue;
              size_t p = lidx(d, G, L, n, m, l);
              for (int b = 0; b < 3; ++b) gmet[(e * L3 + q) * 9 + d + 3 * b] = E.gmet[d][p * 3 + b];
            }
        }
  }
  for (size_t j = 0; j < c.mo.size(); ++j) {
    const Mortar<T> &M = c.mo[j];
    int *t = mortar ? mortar + 17 * j : nullptr;
    if (t) {
      t[0] = M.id[0] + 1; t[1] = M.id[1] + 1; t[2] = M.iface[0]; t[3] = M.iface[1];
      t[4] = M.len[0][0]; t[5] = M.len[1][0]; t[6] = M.len[0][1]; t[7] = M.len[1][1];
      t[8] = M.lenm[0]; t[9] = M.lenm[1]; t[10] = M.orient; t[11] = M.sign; t[12] = M.nsign;
      t[13] = M.conf[0][0]; t[14] = M.conf[1][0]; t[15] = M.conf[0][1]; t[16] = M.conf[1][1];
    }
    for (int jj = 0; jj < M.lenm[1]; ++jj)
      for (int i = 0; i < M.lenm[0]; ++i) {
        size_t q = j * (size_t)ldx * ldx + i + (size_t)ldx * jj;
        if (norm) norm[q] = M.norm[jj * NMX + i];
        if (n_hat)
          for (int k = 0; k < 3; ++k) n_hat[q * 3 + k] = M.n_hat[(jj * NMX + i) * 3 + k];
      }
  }
}

template <class T> Case<T> *from_desc(int ngrid, int nmort, int ldx, const int *ncg, const double *jacob,
                                      const double *gmetg, const double *gmet, const int *mortar,
                                      const double *n_hat, const double *norm) {
  auto *c = new Case<T>();
  rkcoefs(*c, 4);
  const size_t L3 = (size_t)ldx * ldx * ldx;
  c->el.resize(ngrid);
  for (int e = 0; e < ngrid; ++e) {
    Elem<T> &E = c->el[e];
    E.G = ncg[3 * e];
    E.L = E.G + 1;
    const int G = E.G, L = E.L;
    const size_t ng = E.ng(), nl = E.nl();
    E.jacob.resize(ng);
    E.gmetg.resize(9 * ng);
    E.hdelta.resize(ng);
    for (int d = 0; d < 3; ++d) E.gmet[d].resize(3 * nl);
    for (int l = 0; l < L; ++l)
      for (int m = 0; m < L; ++m)
        for (int n = 0; n < L; ++n) {
          size_t q = n + (size_t)ldx * (m + (size_t)ldx * l);
          if (n < G && m < G && l < G) {
            size_t p = gidx(G, n, m, l);
            E.jacob[p] = jacob[e * L3 + q];
            for (int k = 0; k < 9; ++k) E.gmetg[p * 9 + k] = gmetg[(e * L3 + q) * 9 + k];
          }
          for (int d = 0; d < 3; ++d) {
            int idx3[3] = {n, m, l};
            bool ok = true;
            for (int a = 0; a < 3; ++a)
              if (idx3[a] >= (a == d ? L : G)) ok = false;
            if (!ok) continue;
            size_t p = lidx(d, G, L, n, m, l);
            for (int b = 0; b < 3; ++b) E.gmet[d][p * 3 + b] = gmet[(e * L3 + q) * 9 + d + 3 * b];
          }
        }
    for (size_t p = 0; p < ng; ++p)
      E.hdelta[p] = std::pow(std::fabs(1.0 / E.jacob[p]), 1.0 / 3.0) / std::pow((double)(G * G * G), 1.0 / 3.0);
    E.Q.assign(NV * ng, T(0.0));
    E.gQ.assign(NV * ng, T(0.0));
    E.ducros.assign(ng, T(0.0));
    E.rhos.assign(ng, T(0.0));
  }
  c->mo.resize(nmort);
  for (int j = 0; j < nmort; ++j) {
    Mortar<T> &M = c->mo[j];
    const int *t = mortar + 17 * j;
    M.id[0] = t[0] - 1; M.id[1] = t[1] - 1; M.iface[0] = t[2]; M.iface[1] = t[3];
    M.len[0][0] = t[4]; M.len[1][0] = t[5]; M.len[0][1] = t[6]; M.len[1][1] = t[7];
    M.lenm[0] = t[8]; M.lenm[1] = t[9]; M.orient = t[10]; M.sign = t[11]; M.nsign = t[12];
    M.conf[0][0] = t[13]; M.conf[1][0] = t[14]; M.conf[0][1] = t[15]; M.conf[1][1] = t[16];
    M.n_hat.assign(NMX * NMX * 3, 0.0);
    M.norm.assign(NMX * NMX, 0.0);
    for (int jj = 0; jj < M.lenm[1]; ++jj)
      for (int i = 0; i < M.lenm[0]; ++i) {
        size_t q = j * (size_t)ldx * ldx + i + (size_t)ldx * jj;
        M.norm[jj * NMX + i] = norm[q];
        for (int k = 0; k < 3; ++k) M.n_hat[(jj * NMX + i) * 3 + k] = n_hat[q * 3 + k];
      }
    set_mortar_matrices(M);
  }
  return c;
}

// exactsol (caseFiles/tgv/BackstepProblem-stoch.f90:1533-1570) via initc (:1275-1326)
template <class T> void init_tgv(Case<T> &c, double twall, double V0) {
  for (auto &E : c.el) {
    const size_t ng = E.ng();
    for (size_t p = 0; p < ng; ++p) {
      double x = E.xg[3 * p], y = E.xg[3 * p + 1], z = E.xg[3 * p + 2];
      double uu = V0 * std::sin(x) * std::cos(y) * std::cos(z);
      double vv = -V0 * std::cos(x) * std::sin(y) * std::cos(z);
      double ww = 0.0;
      double rho1 = 1.0;
      double pp = twall * rho1 / c.gamma + (std::cos(2.0 * x) + std::cos(2.0 * y)) * (std::cos(2.0 * z) + 2.0) / 16.0;
      double rho = rho1;
      double q[5] = {rho, rho * uu, rho * vv, rho * ww,
                     pp / (c.gamma - 1.0) + 0.5 * rho * (uu * uu + vv * vv + ww * ww)};
      for (int v = 0; v < NV; ++v) E.Q[v * ng + p] = T(q[v] / E.jacob[p]);  // 3DDriver_parfmdf.f90:290-300
    }
  }
}

// dtcalc (Parabolic3D/NS/NS/stac3m/dtcalc.f90:9-58)
template <class T> double dtcalc(const Case<T> &c) {
  double dt = HUGE_VAL;
  for (const auto &E : c.el) {
    const Ops &o = ops_for(E.G);
    const int G = E.G, L = E.L;
    const size_t ng = E.ng();
    for (int l = 0; l < G; ++l) {
      double dcz = o.cx[l + 1] - o.cx[l];
      for (int m = 0; m < G; ++m) {
        double dcy = o.cx[m + 1] - o.cx[m];
        for (int n = 0; n < G; ++n) {
          double dcx = o.cx[n + 1] - o.cx[n];
          size_t p = gidx(G, n, m, l);
          double q1 = re_(E.Q[p]);
          double u0 = std::fabs(re_(E.Q[ng + p]) / q1), v0 = std::fabs(re_(E.Q[2 * ng + p]) / q1),
                 w0 = std::fabs(re_(E.Q[3 * ng + p]) / q1);
          double pp = (c.gamma - 1.0) * (re_(E.Q[4 * ng + p]) - 0.5 * q1 * (u0 * u0 + v0 * v0 + w0 * w0));
          double a = std::sqrt(c.gamma * pp / q1);
          const double *g0 = &E.gmet[0][lidx(0, G, L, n, m, l) * 3];
          const double *g1 = &E.gmet[1][lidx(1, G, L, n, m, l) * 3];
          const double *g2 = &E.gmet[2][lidx(2, G, L, n, m, l) * 3];
          double uu = (u0 + a) * g0[0] + (v0 + a) * g0[1] + (w0 + a) * g0[2];
          double vv = (u0 + a) * g1[0] + (v0 + a) * g1[1] + (w0 + a) * g1[2];
          double ww = (u0 + a) * g2[0] + (v0 + a) * g2[1] + (w0 + a) * g2[2];
          double xl = std::fabs(uu * E.jacob[p]), yl = std::fabs(vv * E.jacob[p]), zl = std::fabs(ww * E.jacob[p]);
          double dti = xl / dcx + yl / dcy + zl / dcz + 1.0e-14;
          dt = std::min(dt, 1.0 / dti);
        }
      }
    }
  }
  return dt;
}

// KE weights bmatu1b (BackstepProblem-stoch.f90:344-361)
void ke_weights(int G, double *bm) {
  const Ops &o = ops_for(G);
  std::vector<double> x(G), w(G);
  gauss_legendre(G, x.data(), w.data());
  for (int i = 0; i < G; ++i)
    for (int j = 0; j < G; ++j)
      for (int l = 0; l < G; ++l) {
        double s = 0.0;
        for (int k = 0; k < G; ++k)
          for (int m = 0; m < G; ++m)
            for (int n = 0; n < G; ++n) {
              double hl = polyn(l, 0.5 * (x[n] + 1.0), G, o.cxg.data());
              double hj = polyn(j, 0.5 * (x[m] + 1.0), G, o.cxg.data());
              double hi = polyn(i, 0.5 * (x[k] + 1.0), G, o.cxg.data());
              s = s + 0.1250 * w[k] * w[m] * w[n] * hi * hj * hl;
            }
        bm[i + G * (j + G * l)] = s;
      }
}

// do_user_stuff KE (BackstepProblem-stoch.f90:463-709) and energydissipation
// (Energydissipation/energydissipation.f90:2-89).
template <class T> void diag(Case<T> &c, double dt, int first, double *turbk, double *dissp, double *enst) {
  std::map<int, std::vector<double>> bms;
  double us = 0, vs = 0, ws = 0;
  for (const auto &E : c.el) {
    auto &bm = bms[E.G];
    if (bm.empty()) {
      bm.resize((size_t)E.G * E.G * E.G);
      ke_weights(E.G, bm.data());
    }
    const int G = E.G;
    const size_t ng = E.ng();
    double su = 0, sv = 0, sw = 0;
    for (int i = 0; i < G; ++i)
      for (int j = 0; j < G; ++j)
        for (int l = 0; l < G; ++l) {
          size_t p = gidx(G, i, j, l);
          double q1 = re_(E.Q[p]);
          double u = re_(E.Q[ng + p]) / q1, v = re_(E.Q[2 * ng + p]) / q1, w = re_(E.Q[3 * ng + p]) / q1;
          double b = bm[i + G * (j + G * l)];
          su = su + (u * u) * b;
          sv = sv + (v * v) * b;
          sw = sw + (w * w) * b;
        }
    us += su;
    vs += sv;
    ws += sw;
  }
  const double j0 = c.el[0].jacob[0];
  us /= j0;
  vs /= j0;
  ws /= j0;
  const double tk = 0.5 * (us + vs + ws) / (8.0 * PI * PI * PI);
  if (first) c.prestep = 0.0;
  *turbk = tk;
  *dissp = (c.prestep - tk) / dt;
  c.prestep = tk;
  // energydissipation
  double sum = 0.0, sum2 = 0.0;
  for (auto &E : c.el) {
    const Ops &o = ops_for(E.G);
    const int G = E.G;
    const size_t ng = E.ng();
    if (!c.ql_valid) continue;
    const T *w3[3] = {E.QL[0].data(), E.QL[1].data(), E.QL[2].data()};
    std::vector<T> gq;
    gauss_deriv(E, o, w3, 4, gq);
    double se = 0.0, sj = 0.0;  // per-element partial sums, then element order
    for (int l = 0; l < G; ++l)
      for (int m = 0; m < G; ++m)
        for (int n = 0; n < G; ++n) {
          size_t p = gidx(G, l, m, n);
          auto Qx = [&](int v) { return re_(gq[(v * 3 + 0) * ng + p]); };
          auto Qy = [&](int v) { return re_(gq[(v * 3 + 1) * ng + p]); };
          auto Qz = [&](int v) { return re_(gq[(v * 3 + 2) * ng + p]); };
          double Q1 = re_(E.Q[p]), Q2 = re_(E.Q[ng + p]), Q3 = re_(E.Q[2 * ng + p]), Q4 = re_(E.Q[3 * ng + p]);
          double jac = E.jacob[p];
          double udery = ((Qy(1) - (Q2 / Q1) * Qy(0))) / Q1;
          double uderz = ((Qz(1) - (Q2 / Q1) * Qz(0))) / Q1;
          double vderx = ((Qx(2) - (Q3 / Q1) * Qx(0))) / Q1;
          double vderz = ((Qz(2) - (Q3 / Q1) * Qz(0))) / Q1;
          double wderx = ((Qx(3) - (Q4 / Q1) * Qx(0))) / Q1;
          double wdery = ((Qy(3) - (Q4 / Q1) * Qy(0))) / Q1;
          double c1 = (wdery - vderz) / jac, c2 = (uderz - wderx) / jac, c3 = (vderx - udery) / jac;
          double vort = c1 * c1 + c2 * c2 + c3 * c3;
          vort = vort / jac;
          sj = sj + 1.0 / jac;
          se = se + vort;
        }
    sum += se;
    sum2 += sj;
  }
  *enst = sum2 > 0 ? 100.0 * (sum / sum2) * (1.0 / c.re) : 0.0;
}

// Enstrophy dissipation of energydissipation (energydissipation.f90:19-78), the
// eps of diag() in the case's scalar type (complex-step derivatives).
template <class T> T enst_t(Case<T> &c) {
  T sum = T(0.0);
  double sum2 = 0.0;
  for (auto &E : c.el) {
    const Ops &o = ops_for(E.G);
    const int G = E.G;
    const size_t ng = E.ng();
    if (!c.ql_valid) continue;
    const T *w3[3] = {E.QL[0].data(), E.QL[1].data(), E.QL[2].data()};
    std::vector<T> gq;
    gauss_deriv(E, o, w3, 4, gq);
    T se = T(0.0);
    double sj = 0.0;
    for (int l = 0; l < G; ++l)
      for (int m = 0; m < G; ++m)
        for (int n = 0; n < G; ++n) {
          size_t p = gidx(G, l, m, n);
          auto Qx = [&](int v) { return gq[(v * 3 + 0) * ng + p]; };
          auto Qy = [&](int v) { return gq[(v * 3 + 1) * ng + p]; };
          auto Qz = [&](int v) { return gq[(v * 3 + 2) * ng + p]; };
          T Q1 = E.Q[p], Q2 = E.Q[ng + p], Q3 = E.Q[2 * ng + p], Q4 = E.Q[3 * ng + p];
          double jac = E.jacob[p];
          T udery = ((Qy(1) - (Q2 / Q1) * Qy(0))) / Q1;
          T uderz = ((Qz(1) - (Q2 / Q1) * Qz(0))) / Q1;
          T vderx = ((Qx(2) - (Q3 / Q1) * Qx(0))) / Q1;
          T vderz = ((Qz(2) - (Q3 / Q1) * Qz(0))) / Q1;
          T wderx = ((Qx(3) - (Q4 / Q1) * Qx(0))) / Q1;
          T wdery = ((Qy(3) - (Q4 / Q1) * Qy(0))) / Q1;
          T c1 = (wdery - vderz) / jac, c2 = (uderz - wderx) / jac, c3 = (vderx - udery) / jac;
          T vort = c1 * c1 + c2 * c2 + c3 * c3;
          vort = vort / jac;
          sj = sj + 1.0 / jac;
          se = se + vort;
        }
    sum += se;
    sum2 += sj;
  }
  return sum2 > 0 ? 100.0 * (sum / sum2) * (1.0 / c.re) : T(0.0);
}

// The case with its state in another scalar type (geometry and parameters copied).
template <class T> Case<T> *convert_case(const Case<double> &c) {
  auto *o = new Case<T>();
  auto cv = [](const std::vector<double> &a) { return std::vector<T>(a.begin(), a.end()); };
  o->el.resize(c.el.size());
  for (size_t e = 0; e < c.el.size(); ++e) {
    const auto &A = c.el[e];
    auto &B = o->el[e];
    B.G = A.G;
    B.L = A.L;
    std::memcpy(B.corner, A.corner, sizeof(A.corner));
    std::memcpy(B.node, A.node, sizeof(A.node));
    std::memcpy(B.mort, A.mort, sizeof(A.mort));
    std::memcpy(B.mside, A.mside, sizeof(A.mside));
    std::memcpy(B.orientation, A.orientation, sizeof(A.orientation));
    std::memcpy(B.boundary, A.boundary, sizeof(A.boundary));
    B.jacob = A.jacob;
    B.gmetg = A.gmetg;
    for (int d = 0; d < 3; ++d) B.gmet[d] = A.gmet[d];
    B.xg = A.xg;
    B.hdelta = A.hdelta;
    B.Q = cv(A.Q);
    B.gQ = cv(A.gQ);
    for (int d = 0; d < 3; ++d) {
      B.QL[d] = cv(A.QL[d]);
      B.F[d] = cv(A.F[d]);
      B.R[d] = cv(A.R[d]);
      B.muh[d] = cv(A.muh[d]);
      B.nut[d] = cv(A.nut[d]);
    }
    B.muhg = cv(A.muhg);
    B.nutg = cv(A.nutg);
    B.ducros = cv(A.ducros);
    B.rhos = cv(A.rhos);
  }
  o->mo.resize(c.mo.size());
  for (size_t j = 0; j < c.mo.size(); ++j) {
    const auto &A = c.mo[j];
    auto &B = o->mo[j];
    std::memcpy(B.id, A.id, sizeof(A.id));
    std::memcpy(B.iface, A.iface, sizeof(A.iface));
    std::memcpy(B.len, A.len, sizeof(A.len));
    std::memcpy(B.lenm, A.lenm, sizeof(A.lenm));
    B.orient = A.orient;
    B.sign = A.sign;
    B.nsign = A.nsign;
    std::memcpy(B.conf, A.conf, sizeof(A.conf));
    B.n_hat = A.n_hat;
    B.norm = A.norm;
    for (int a = 0; a < 2; ++a)
      for (int d = 0; d < 2; ++d) {
        B.P[a][d] = A.P[a][d];
        B.Rm[a][d] = A.Rm[a][d];
        B.pin[a][d] = A.pin[a][d];
      }
    for (int a = 0; a < 2; ++a) {
      B.Qm[a] = cv(A.Qm[a]);
      B.fv[a] = cv(A.fv[a]);
    }
    B.bc = A.bc;  // boundary mortars: condition and external states
    B.Qx = A.Qx;
    B.fvx = A.fvx;
  }
  o->gamma = c.gamma;
  o->re = c.re;
  o->pr = c.pr;
  o->mach = c.mach;
  o->twall = c.twall;
  o->cmu = c.cmu;
  o->mumax = c.mumax;
  o->shock = c.shock;
  o->ducros = c.ducros;
  o->les = c.les;
  o->shock_sensor = c.shock_sensor;
  o->rho_sensor = c.rho_sensor;
  o->cs = c.cs;
  o->numax = c.numax;
  o->iord = c.iord;
  o->kord = c.kord;
  std::memcpy(o->ark, c.ark, sizeof(c.ark));
  std::memcpy(o->brk, c.brk, sizeof(c.brk));
  std::memcpy(o->crk, c.crk, sizeof(c.crk));
  o->ql_valid = c.ql_valid;
  o->prestep = c.prestep;
  return o;
}

}  // namespace

// ====================================================================== C API
struct orc_case {
  Case<double> *c;
};

extern "C" {

orc_case *orc_build_box(int nex, int ney, int nez, double lx, double ly, double lz, const int *orders, const int *rot) {
  auto *h = new orc_case;
  h->c = build_box<double>(nex, ney, nez, lx, ly, lz, orders, rot);
  return h;
}
orc_case *orc_from_desc(int ngrid, int nmort, int ldx, const int *ncg, const double *jacob, const double *gmetg,
                        const double *gmet, const int *mortar, const double *n_hat, const double *norm) {
  auto *h = new orc_case;
  h->c = from_desc<double>(ngrid, nmort, ldx, ncg, jacob, gmetg, gmet, mortar, n_hat, norm);
  return h;
}
void orc_free(orc_case *h) {
  if (!h) return;
  delete h->c;
  delete h;
}
void orc_set_phys(orc_case *h, double gamma, double re, double pr, double mach, double cmu, double mumax, int shock,
                  int iord) {
  auto &c = *h->c;
  c.gamma = gamma;
  c.re = re;
  c.pr = pr;
  c.mach = mach;
  c.cmu = cmu;
  c.mumax = mumax;
  c.shock = shock != 0;
  c.ducros = (shock & 2) != 0;
  rkcoefs(c, iord);
  if (c.shock)
    for (auto &E : c.el) {
      E.muhg.assign(E.ng(), 0.0);
      for (int d = 0; d < 3; ++d) E.muh[d].assign(E.nl(), 0.0);
    }
}
// d%bcond of every element face ([ngrid][6], BC_* codes); boundary mortars
// (id(2) = 0) take the code of their master face
int orc_set_bcond(orc_case *h, const int *bcond) {
  auto &c = *h->c;
  for (size_t e = 0; e < c.el.size(); ++e)
    for (int f = 0; f < 6; ++f) c.el[e].bcond[f] = bcond[6 * e + f];
  for (auto &M : c.mo) {
    if (M.id[1] >= 0) continue;
    M.bc = c.el[M.id[0]].bcond[M.iface[0] - 1];
    if (M.bc < BC_WALLADIAB || M.bc > BC_OUTFLOW) return -1;
  }
  return 0;
}
// twall and the external mrtr%Q(:,:,:,2) / mrtr%fv(:,:,:,2) of the boundary
// mortars ([nmort][5][ldx][ldx], i fastest; a null array keeps the previous
// values, zero initially)
void orc_set_boundary(orc_case *h, double twall, const double *Qx, const double *fvx, int ldx) {
  auto &c = *h->c;
  c.twall = twall;
  for (size_t j = 0; j < c.mo.size(); ++j) {
    auto &M = c.mo[j];
    if (M.id[1] >= 0) continue;
    if (M.Qx.empty()) M.Qx.assign(NV * NMX * NMX, 0.0);  // a null array keeps the previous state
    if (M.fvx.empty()) M.fvx.assign(NV * NMX * NMX, 0.0);
    for (int v = 0; v < NV; ++v)
      for (int jj = 0; jj < M.lenm[1]; ++jj)
        for (int i = 0; i < M.lenm[0]; ++i) {
          const size_t q = (((size_t)j * NV + v) * ldx + jj) * ldx + i;
          if (Qx) M.Qx[v * NMX * NMX + jj * NMX + i] = Qx[q];
          if (fvx) M.fvx[v * NMX * NMX + jj * NMX + i] = fvx[q];
        }
  }
}
int orc_nel(const orc_case *h) { return (int)h->c->el.size(); }
int orc_nmort(const orc_case *h) { return (int)h->c->mo.size(); }
int orc_ncg(const orc_case *h, int e) { return h->c->el[e].G; }
void orc_export_desc(const orc_case *h, int ldx, int *ncg, double *jacob, double *gmetg, double *gmet, int *mortar,
                     double *n_hat, double *norm, double *xg) {
  export_desc(*h->c, ldx, ncg, jacob, gmetg, gmet, mortar, n_hat, norm, xg);
}
void orc_operators(int p, double *dmx, double *bx) {
  const Ops &o = ops_for(p + 1);
  std::memcpy(dmx, o.dmx.data(), sizeof(double) * o.dmx.size());
  std::memcpy(bx, o.bx.data(), sizeof(double) * o.bx.size());
}
void orc_projection(int nin, int nout, double *prolong, double *restrict_) {
  std::vector<double> ci(nin), co(nout);
  gauss_points(nin, ci.data());
  gauss_points(nout, co.data());
  compute_pmat(ci.data(), nin, co.data(), nout, prolong);
  compute_pmat(co.data(), nout, ci.data(), nin, restrict_);
}
void orc_ke_weights(int G, double *w) { ke_weights(G, w); }
void orc_init_tgv(orc_case *h, double twall, double v0) {
  if (h->c->el[0].xg.empty()) return;
  init_tgv(*h->c, twall, v0);
}
void orc_set_q(orc_case *h, const double *JQ, int ldx) {
  const size_t L3 = (size_t)ldx * ldx * ldx;
  for (size_t e = 0; e < h->c->el.size(); ++e) {
    auto &E = h->c->el[e];
    const int G = E.G;
    const size_t ng = E.ng();
    for (int v = 0; v < NV; ++v)
      for (int l = 0; l < G; ++l)
        for (int m = 0; m < G; ++m)
          for (int n = 0; n < G; ++n)
            E.Q[v * ng + gidx(G, n, m, l)] = JQ[e * NV * L3 + n + (size_t)ldx * (m + (size_t)ldx * (l + (size_t)ldx * v))];
  }
}
void orc_get_q(const orc_case *h, double *JQ, int ldx) {
  const size_t L3 = (size_t)ldx * ldx * ldx;
  for (size_t e = 0; e < h->c->el.size(); ++e) {
    const auto &E = h->c->el[e];
    const int G = E.G;
    const size_t ng = E.ng();
    for (int v = 0; v < NV; ++v)
      for (int l = 0; l < G; ++l)
        for (int m = 0; m < G; ++m)
          for (int n = 0; n < G; ++n)
            JQ[e * NV * L3 + n + (size_t)ldx * (m + (size_t)ldx * (l + (size_t)ldx * v))] = E.Q[v * ng + gidx(G, n, m, l)];
  }
}
// Lobatto arrays of the last Fluxes call (d%Qlgg, d%Qglg, d%Qggl, the arrays
// write_restart stores: Parabolic3D/stac3m/restart.f90:116-118), in DSEM's
// DIMENSION(nx,ny,nz,neq) layout with nx = ny = nz = ldx: out[e][grid d][v][ldx^3],
// grid d having L = G+1 points along d; padding left zero.  Returns 0 when the
// arrays were never computed (DSEM's zeroed arrays).
int orc_get_lobatto(const orc_case *h, double *out, int ldx) {
  const size_t L3 = (size_t)ldx * ldx * ldx;
  std::fill(out, out + h->c->el.size() * 3 * NV * L3, 0.0);
  if (!h->c->ql_valid) return 0;
  for (size_t e = 0; e < h->c->el.size(); ++e) {
    const auto &E = h->c->el[e];
    const int G = E.G, L = E.L;
    const size_t nl = E.nl();
    for (int d = 0; d < 3; ++d) {
      const int ex = d == 0 ? L : G, ey = d == 1 ? L : G, ez = d == 2 ? L : G;
      for (int v = 0; v < NV; ++v)
        for (int z = 0; z < ez; ++z)
          for (int y = 0; y < ey; ++y)
            for (int x = 0; x < ex; ++x)
              out[((e * 3 + d) * NV + v) * L3 + x + (size_t)ldx * (y + (size_t)ldx * z)] =
                  re_(E.QL[d][v * nl + x + (size_t)ex * (y + (size_t)ey * z)]);
    }
  }
  return 1;
}
double orc_dtcalc(const orc_case *h) { return dtcalc(*h->c); }
void orc_rhs(orc_case *h, double tk, double *Qt, int ldx) {
  (void)tk;
  fluxes(*h->c);
  update_all(*h->c, 0.0, 0, Qt, ldx);
}
int orc_stage(orc_case *h, double time, double dt, int kk, double *Qt, int ldx) {
  return stage(*h->c, time, dt, kk, Qt, ldx);
}
int orc_step(orc_case *h, double time, double dt, int nsteps) {
  auto &c = *h->c;
  for (int s = 0; s < nsteps; ++s) {
    for (int kk = 1; kk <= c.kord; ++kk) {
      int st = stage(c, time + dt * c.brk[kk - 1], dt, kk, nullptr, 0);
      if (st) return st;
    }
    time += dt;
  }
  return 0;
}
void orc_diag(orc_case *h, double dt, int first, double *turbk, double *dissp, double *enst) {
  diag(*h->c, dt, first, turbk, dissp, enst);
}
void orc_get_muhg(const orc_case *h, double *mu, int ldx) {
  for (size_t e = 0; e < h->c->el.size(); ++e) {
    const auto &E = h->c->el[e];
    const int G = E.G;
    for (int l = 0; l < G; ++l)
      for (int m = 0; m < G; ++m)
        for (int n = 0; n < G; ++n)
          mu[e * (size_t)ldx * ldx * ldx + n + (size_t)ldx * (m + (size_t)ldx * l)] =
              E.muhg.empty() ? 0.0 : E.muhg[gidx(G, n, m, l)];
  }
}
int orc_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
#else
  (void)n;
  return 1;
#endif
}
int orc_kord(const orc_case *h) { return h->c->kord; }
void orc_riemann(const double *nh, double ds, const double *Ql, const double *Qr, double gamma, double *flux) {
  riemann(nh, ds, Ql, Qr, gamma, flux);
}
void orc_euler(const double *Q, double gamma, double *f, double *g, double *h) { euler_fluxes(Q, gamma, f, g, h); }
void orc_vis(const double *Q, const double *Qx, const double *Qy, const double *Qz, double amu, double gamma,
             double pr, double mach, double *f, double *g, double *h) {
  vis_fluxes(Q, Qx, Qy, Qz, amu, gamma, pr, mach, f, g, h);
}
// J = sum over the last `window` of `nsteps` steps of dt * eps_n (eps_n = the
// enstrophy dissipation of orc_diag after step n), from the current state
// plus i*hstep*dq (complex step): *J = Re J, *dJ = Im J / hstep = dJ/dJQ . dq.
// The case itself is left unchanged.  dq uses the ldx layout of orc_set_q.
void orc_objective_cs(const orc_case *h, double dt, int nsteps, int window, const double *dq, double hstep, int ldx,
                      double *J, double *dJ) {
  using CT = std::complex<double>;
  Case<CT> *cc = convert_case<CT>(*h->c);
  const size_t L3 = (size_t)ldx * ldx * ldx;
  if (dq)
    for (size_t e = 0; e < cc->el.size(); ++e) {
      auto &E = cc->el[e];
      const int G = E.G;
      const size_t ng = E.ng();
      for (int v = 0; v < NV; ++v)
        for (int l = 0; l < G; ++l)
          for (int m = 0; m < G; ++m)
            for (int n = 0; n < G; ++n) {
              CT &q = E.Q[v * ng + gidx(G, n, m, l)];
              q = CT(q.real(), hstep * dq[e * NV * L3 + n + (size_t)ldx * (m + (size_t)ldx * (l + (size_t)ldx * v))]);
            }
    }
  CT Jc = 0.0;
  for (int s = 0; s < nsteps; ++s) {
    for (int kk = 1; kk <= cc->kord; ++kk) stage(*cc, 0.0, dt, kk, nullptr, 0);
    if (s >= nsteps - window) Jc += dt * enst_t(*cc);
  }
  *J = Jc.real();
  *dJ = hstep != 0.0 ? Jc.imag() / hstep : 0.0;
  delete cc;
}
void orc_set_les(orc_case *h, double cs, double numax) {
  auto &c = *h->c;
  c.les = cs > 0.0;
  c.cs = cs;
  c.numax = numax;
  for (auto &E : c.el) {
    E.nutg.assign(E.ng(), 0.0);
    for (int d = 0; d < 3; ++d) E.nut[d].assign(E.nl(), 0.0);
  }
}
void orc_set_les_sensors(orc_case *h, int shock_sensor, int rho_sensor) {
  h->c->shock_sensor = shock_sensor != 0;
  h->c->rho_sensor = rho_sensor != 0;
}
void orc_get_nut(const orc_case *h, double *nu, int ldx) {
  for (size_t e = 0; e < h->c->el.size(); ++e) {
    const auto &E = h->c->el[e];
    const int G = E.G;
    for (int l = 0; l < G; ++l)
      for (int m = 0; m < G; ++m)
        for (int n = 0; n < G; ++n)
          nu[e * (size_t)ldx * ldx * ldx + n + (size_t)ldx * (m + (size_t)ldx * l)] =
              E.nutg.empty() ? 0.0 : E.nutg[gidx(G, n, m, l)];
  }
}
void orc_rk(const orc_case *h, double *a, double *b, double *c) {
  for (int i = 0; i < 5; ++i) {
    a[i] = h->c->ark[i];
    b[i] = h->c->brk[i];
    c[i] = h->c->crk[i];
  }
}

}  // extern "C"
