// dsem_host_math.h -- host-side spectral setup: Chebyshev Gauss / Lobatto
// points, Lagrange derivative and interpolation matrices, Gauss-Legendre
// quadrature, L2 mortar projections and the kinetic-energy quadrature weights.
//
// These restate set_points (Grid_Routines/stac3m_geomLib.f90:7-75), polyn /
// polynder (Independentroutines/baselib.f90:18-80), dermat / intrpmat
// (Spectral/stac3m/matrices.f90:144-207), compute_pmat
// (Spectral/mortarLib.f90:242-420) and bmatu1b
// (caseFiles/tgv/BackstepProblem-stoch.f90:344-361); the arithmetic order is
// DSEM's, so the matrices are reproducible bit for bit on one host.
#pragma once
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <vector>

namespace dsem {
namespace hostmath {

constexpr double PI = 3.141592653589793238462643;

inline double polyn(int k, double x, int n, const double *z) {
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

inline double polynder(int k, double x, int n, const double *z) {
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

inline void lobatto_points(int L, double *cx) {
  for (int n = 0; n < L; ++n) cx[n] = 0.5 * (1.0 - std::cos((double)n * PI / (double)(L - 1)));
}
inline void gauss_points(int G, double *cxg) {
  for (int n = 1; n <= G; ++n) cxg[n - 1] = 0.5 * (1.0 - std::cos((2.0 * n - 1.0) * PI / (2.0 * ((double)G - 1.0) + 2.0)));
}

// dmx [G][L] (derivative of Lobatto Lagrange polynomials at Gauss points,
// diagonal set by the negative row sum) and bx [L][G] (Gauss Lagrange
// polynomials at Lobatto points).
inline void operators(int G, double *dmx, double *bx) {
  const int L = G + 1;
  std::vector<double> cx(L), cxg(G);
  lobatto_points(L, cx.data());
  gauss_points(G, cxg.data());
  for (int i = 0; i < G * L; ++i) dmx[i] = 0.0;
  for (int k = 0; k < G; ++k) {
    double sum = 0.0;
    for (int j = 0; j < L; ++j) {
      if (j == k) continue;
      double b = polynder(j, cxg[k], L, cx.data());
      if (std::fabs(b) < DBL_EPSILON) b = 0.0;
      dmx[k * L + j] = b;
      sum = sum - b;
      dmx[k * L + k] = sum;
    }
  }
  for (int n = 0; n < L; ++n)
    for (int j = 0; j < G; ++j) bx[n * G + j] = polyn(j, cx[n], G, cxg.data());
}

// Gauss-Legendre nodes (ascending) and weights on [-1,1], by Newton iteration
// on the Legendre recurrence (Golub-Welsch in DSEM; any accurate method).
inline void gauss_legendre(int n, double *x, double *w) {
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

// L2 projection from nodes cxin (ni) to nodes cxo (no): out [no][ni]
inline void projection(const double *cxin, int ni, const double *cxo, int no, double *pmat) {
  const int nmx = std::max(ni, no);
  std::vector<double> xg(nmx), wg(nmx);
  gauss_legendre(no, xg.data(), wg.data());
  std::vector<double> bm(no * no), am(no * ni);
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
  gauss_legendre(nmx, xg.data(), wg.data());
  for (int i = 0; i < no; ++i)
    for (int j = 0; j < ni; ++j) {
      double s = 0.0;
      for (int k = 0; k < nmx; ++k) {
        double xi = 0.5 * (xg[k] + 1.0);
        s = s + 0.5 * wg[k] * polyn(j, xi, ni, cxin) * polyn(i, xi, no, cxo);
      }
      am[i + no * j] = s;
    }
  // Gaussian elimination with partial pivoting, then back substitution per column
  std::vector<int> piv(no);
  for (int k = 0; k < no; ++k) {
    int p = k;
    for (int i = k + 1; i < no; ++i)
      if (std::fabs(bm[i + no * k]) > std::fabs(bm[p + no * k])) p = i;
    piv[k] = p;
    if (p != k)
      for (int j = 0; j < no; ++j) std::swap(bm[k + no * j], bm[p + no * j]);
    for (int i = k + 1; i < no; ++i) {
      bm[i + no * k] /= bm[k + no * k];
      for (int j = k + 1; j < no; ++j) bm[i + no * j] -= bm[i + no * k] * bm[k + no * j];
    }
  }
  for (int c = 0; c < ni; ++c) {
    double *b = &am[(size_t)no * c];
    for (int k = 0; k < no; ++k) {
      std::swap(b[k], b[piv[k]]);
      for (int i = k + 1; i < no; ++i) b[i] -= bm[i + no * k] * b[k];
    }
    for (int k = no - 1; k >= 0; --k) {
      for (int j = k + 1; j < no; ++j) b[k] -= bm[k + no * j] * b[j];
      b[k] /= bm[k + no * k];
    }
  }
  for (int i = 0; i < no; ++i)
    for (int j = 0; j < ni; ++j) {
      double v = am[i + no * j];
      pmat[i * ni + j] = std::fabs(v) <= 100 * DBL_EPSILON ? 0.0 : v;
    }
}

// kinetic-energy quadrature weights w[i + G*(j + G*l)]
inline void ke_weights(int G, double *bm) {
  std::vector<double> x(G), w(G), cxg(G);
  gauss_points(G, cxg.data());
  gauss_legendre(G, x.data(), w.data());
  for (int i = 0; i < G; ++i)
    for (int j = 0; j < G; ++j)
      for (int l = 0; l < G; ++l) {
        double s = 0.0;
        for (int k = 0; k < G; ++k)
          for (int m = 0; m < G; ++m)
            for (int n = 0; n < G; ++n) {
              double hl = polyn(l, 0.5 * (x[n] + 1.0), G, cxg.data());
              double hj = polyn(j, 0.5 * (x[m] + 1.0), G, cxg.data());
              double hi = polyn(i, 0.5 * (x[k] + 1.0), G, cxg.data());
              s = s + 0.1250 * w[k] * w[m] * w[n] * hi * hj * hl;
            }
        bm[i + G * (j + G * l)] = s;
      }
}

}  // namespace hostmath
}  // namespace dsem
