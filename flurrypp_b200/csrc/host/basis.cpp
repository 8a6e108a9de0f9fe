// 1-D point sets, Lagrange/Legendre/VCJH polynomials and the dense FR
// operator matrices (reference: src/points.cpp, src/polynomials.cpp,
// src/operators.cpp:46-1001, 1449-1506, 1552-1634).
//
// Gauss-Legendre and Gauss-Lobatto nodes and Gauss weights are computed here
// by Newton iteration in long double (the reference tabulates them to 15
// digits, points.cpp:198-403, 405-470); the two agree to <= 5e-16.
#include <algorithm>
#include <cmath>

#include "fr_host.hpp"

namespace fr {

namespace {

// P_n(x) and P_n'(x) by the three-term recurrence, long double.
void legendre_ld(int n, long double x, long double &p, long double &dp) {
  long double p0 = 1.0L, p1 = x;
  if (n == 0) {
    p = 1.0L;
    dp = 0.0L;
    return;
  }
  for (int k = 2; k <= n; k++) {
    long double pk = ((2 * k - 1) * x * p1 - (k - 1) * p0) / k;
    p0 = p1;
    p1 = pk;
  }
  p = p1;
  dp = n * (x * p1 - p0) / (x * x - 1.0L);
}

std::vector<long double> gauss_legendre_nodes(int n) {
  std::vector<long double> x(n);
  const long double PI = 3.141592653589793238462643383279502884L;
  for (int i = 0; i < n; i++) {
    long double z = std::cos(PI * (i + 0.75L) / (n + 0.5L));
    for (int it = 0; it < 100; it++) {
      long double p, dp;
      legendre_ld(n, z, p, dp);
      long double dz = p / dp;
      z -= dz;
      if (std::fabs(dz) < 1e-19L) break;
    }
    x[i] = z;
  }
  std::sort(x.begin(), x.end());
  for (int i = 0; i < n / 2; i++) {  // exact symmetry
    long double m = 0.5L * (x[n - 1 - i] - x[i]);
    x[i] = -m;
    x[n - 1 - i] = m;
  }
  if (n % 2) x[n / 2] = 0.0L;
  return x;
}

// Interior Gauss-Lobatto nodes: roots of P_{n-1}'(x), with x = +-1 added.
std::vector<long double> gauss_lobatto_nodes(int n) {
  std::vector<long double> x(n);
  if (n == 1) {
    x[0] = 0.0L;
    return x;
  }
  const long double PI = 3.141592653589793238462643383279502884L;
  int N = n - 1;
  x[0] = -1.0L;
  x[n - 1] = 1.0L;
  for (int i = 1; i < n - 1; i++) {
    long double z = -std::cos(PI * i / N);
    for (int it = 0; it < 100; it++) {
      // f = P_N'(z), f' = P_N''(z) = (2 z P_N' - N(N+1) P_N) / (1 - z^2)
      long double p, dp;
      legendre_ld(N, z, p, dp);
      long double d2p = (2.0L * z * dp - N * (N + 1) * p) / (1.0L - z * z);
      long double dz = dp / d2p;
      z -= dz;
      if (std::fabs(dz) < 1e-19L) break;
    }
    x[i] = z;
  }
  std::sort(x.begin(), x.end());
  for (int i = 0; i < n / 2; i++) {
    long double m = 0.5L * (x[n - 1 - i] - x[i]);
    x[i] = -m;
    x[n - 1 - i] = m;
  }
  if (n % 2) x[n / 2] = 0.0L;
  return x;
}

}  // namespace

std::vector<double> pts1d(int ptsType, int order) {
  int n = order + 1;
  std::vector<double> out(n);
  if (ptsType == PTS_EQUIDISTANT) {
    double dxi = 2.0 / order;
    for (int i = 0; i < n; i++) out[i] = -1 + dxi * i;
    return out;
  }
  auto x = ptsType == PTS_LOBATTO ? gauss_lobatto_nodes(n) : gauss_legendre_nodes(n);
  for (int i = 0; i < n; i++) out[i] = (double)x[i];
  return out;
}

std::vector<double> qwts1d(int order) {
  int n = order + 1;
  auto x = gauss_legendre_nodes(n);
  std::vector<double> w(n);
  for (int i = 0; i < n; i++) {
    long double p, dp;
    legendre_ld(n, x[i], p, dp);
    w[i] = (double)(2.0L / ((1.0L - x[i] * x[i]) * dp * dp));
  }
  if (n == 1) w[0] = 2.0;
  return w;
}

// reference: src/polynomials.cpp:39-50
double lagrange(const std::vector<double> &x, double y, int mode) {
  double lag = 1.0;
  for (int i = 0; i < (int)x.size(); i++)
    if (i != mode) lag = lag * ((y - x[i]) / (x[mode] - x[i]));
  return lag;
}

// reference: src/polynomials.cpp:53-80
double dlagrange(const std::vector<double> &x, double y, int mode) {
  double d = 0.0;
  int n = (int)x.size();
  for (int i = 0; i < n; i++) {
    if (i == mode) continue;
    double num = 1.0, den = 1.0;
    for (int j = 0; j < n; j++) {
      if (j != mode && j != i) num = num * (y - x[j]);
      if (j != mode) den = den * (x[mode] - x[j]);
    }
    d = d + num / den;
  }
  return d;
}

// reference: src/polynomials.cpp:119-129
double legendre(double r, int n) {
  if (n < 0) return 0.0;
  if (n == 0) return 1.0;
  double p0 = 1.0, p1 = r;
  for (int k = 2; k <= n; k++) {
    double pk = ((2 * k - 1) * r * p1 - (k - 1) * p0) / k;
    p0 = p1;
    p1 = pk;
  }
  return p1;
}

// reference: src/polynomials.cpp:131-151
double dlegendre(double r, int n) {
  if (n == 0) return 0.0;
  if (r > -1.0 && r < 1.0)
    return n * ((r * legendre(r, n)) - legendre(r, n - 1)) / (r * r - 1.0);
  if (r == -1.0) return std::pow(-1.0, n - 1.0) * 0.5 * n * (n + 1.0);
  return 0.5 * n * (n + 1.0);
}

static double factorial_d(int n) { return n <= 1 ? 1.0 : n * factorial_d(n - 1); }

// reference: src/polynomials.cpp:423-460
double compute_eta(int scheme, int order) {
  switch (scheme) {
    case 0:
      return 0.0;
    case 1:
      return (1.0 * order) / (1.0 * (order + 1));
    case 2:
      return (1.0 * (order + 1)) / (1.0 * order);
    case 3: {
      double c1d = order == 2 ? 0.206 : order == 3 ? 3.80e-3 : order == 4 ? 4.67e-5 : 4.28e-7;
      double ap = 1.0 / std::pow(2.0, order) * factorial_d(2 * order) /
                  (factorial_d(order) * factorial_d(order));
      return c1d * (2 * order + 1) / 2 * (factorial_d(order) * ap) * (factorial_d(order) * ap);
    }
  }
  return 0.0;
}

// Derivative of the left (mode 0) / right (mode 1) VCJH correction function
// (reference: src/polynomials.cpp:473-493).
double dvcjh_1d(double r, int mode, int order, double eta) {
  if (mode == 0) {
    if (order == 0)
      return 0.5 * std::pow(-1.0, order) * (dlegendre(r, order) - (dlegendre(r, order + 1) / (1.0 + eta)));
    return 0.5 * std::pow(-1.0, order) *
           (dlegendre(r, order) -
            ((eta * dlegendre(r, order - 1) + dlegendre(r, order + 1)) / (1.0 + eta)));
  }
  if (order == 0) return 0.5 * (dlegendre(r, order) + (dlegendre(r, order + 1) / (1.0 + eta)));
  return 0.5 * (dlegendre(r, order) +
                ((eta * dlegendre(r, order - 1) + dlegendre(r, order + 1)) / (1.0 + eta)));
}

double cfl_limit(int order) {
  static const double lim[] = {1.393, 0.464, 0.235, 0.1453, 0.100, 0.0736};
  return order >= 0 && order <= 5 ? lim[order] : 0.0;
}

// Tensor-product solution points: x fastest (reference: src/points.cpp:67-96).
std::vector<Pt> loc_spts(int nDims, int order, int ptsType) {
  auto p = pts1d(ptsType, order);
  int n = order + 1;
  std::vector<Pt> out;
  if (nDims == 2) {
    out.resize(n * n);
    for (int i = 0; i < n; i++)
      for (int j = 0; j < n; j++) {
        out[j + i * n].x = p[j];
        out[j + i * n].y = p[i];
      }
  } else {
    out.resize(n * n * n);
    for (int k = 0; k < n; k++)
      for (int j = 0; j < n; j++)
        for (int i = 0; i < n; i++) {
          Pt &q = out[i + n * (j + n * k)];
          q.x = p[i];
          q.y = p[j];
          q.z = p[k];
        }
  }
  return out;
}

// Flux points face by face; quads: bottom, right, top, left, counter-clockwise
// (reference: src/points.cpp:100-162); hexes: z-, z+, x-, x+, y-, y+.
std::vector<Pt> loc_fpts(int nDims, int order, int ptsType) {
  auto p = pts1d(ptsType, order);
  int n = order + 1;
  std::vector<Pt> out;
  if (nDims == 2) {
    out.resize(4 * n);
    for (int i = 0; i < n; i++) {
      out[i].x = p[i];
      out[i].y = -1.0;
      out[i + n].x = 1.0;
      out[i + n].y = p[i];
      out[i + 2 * n].x = p[order - i];
      out[i + 2 * n].y = 1.0;
      out[i + 3 * n].x = -1.0;
      out[i + 3 * n].y = p[order - i];
    }
  } else {
    int n2 = n * n;
    out.resize(6 * n2);
    for (int i = 0; i < n; i++)
      for (int j = 0; j < n; j++) {
        int ind = i + j * n;
        out[ind] = {p[i], p[j], -1.0};
        out[ind + n2] = {p[order - i], p[j], 1.0};
        out[ind + 2 * n2] = {-1.0, p[i], p[j]};
        out[ind + 3 * n2] = {1.0, p[order - i], p[j]};
        out[ind + 4 * n2] = {p[order - i], -1.0, p[j]};
        out[ind + 5 * n2] = {p[i], 1.0, p[j]};
      }
  }
  return out;
}

// Gauss weights in solution-point order (reference: src/points.cpp:405-431;
// always Gauss-Legendre weights, whatever the point set).
std::vector<double> spt_weights(int nDims, int order) {
  auto w = qwts1d(order);
  int n = order + 1;
  std::vector<double> out;
  if (nDims == 1) return w;
  if (nDims == 2) {
    out.resize(n * n);
    for (int i = 0; i < n; i++)
      for (int j = 0; j < n; j++) out[j + i * n] = w[i] * w[j];
  } else {
    out.resize(n * n * n);
    for (int i = 0; i < n; i++)
      for (int j = 0; j < n; j++)
        for (int k = 0; k < n; k++) out[k + n * (j + i * n)] = w[i] * w[j] * w[k];
  }
  return out;
}

std::vector<double> face_weights(int nDims, int order) { return spt_weights(nDims - 1, order); }

static void face_normal(int nDims, int iFace, double *t) {
  t[0] = t[1] = t[2] = 0.0;
  if (nDims == 2) {
    static const double q[4][2] = {{0, -1}, {1, 0}, {0, 1}, {-1, 0}};
    t[0] = q[iFace][0];
    t[1] = q[iFace][1];
  } else {
    static const double h[6][3] = {{0, 0, -1}, {0, 0, 1}, {-1, 0, 0},
                                   {1, 0, 0},  {0, -1, 0}, {0, 1, 0}};
    for (int d = 0; d < 3; d++) t[d] = h[iFace][d];
  }
}

void build_operators(int nDims, int order, int ptsType, int vcjh, Operators &op) {
  op.nDims = nDims;
  op.order = order;
  int n = order + 1;
  auto sp = loc_spts(nDims, order, ptsType);
  auto fp = loc_fpts(nDims, order, ptsType);
  auto p1 = pts1d(ptsType, order);
  int nS = (int)sp.size(), nF = (int)fp.size();
  op.nSpts = nS;
  op.nFpts = nF;
  int nPF = nDims == 2 ? n : n * n;

  // spt index -> (i, j, k)
  auto ijk = [&](int s, int &i, int &j, int &k) {
    if (nDims == 2) {
      i = s % n;
      j = s / n;
      k = 0;
    } else {
      k = s / (n * n);
      j = (s - n * n * k) / n;
      i = s - n * j - n * n * k;
    }
  };

  // opp_spts_to_fpts (operators.cpp:112-141)
  op.ext.assign((size_t)nF * nS, 0.0);
  for (int f = 0; f < nF; f++)
    for (int s = 0; s < nS; s++) {
      int i, j, k;
      ijk(s, i, j, k);
      double v = lagrange(p1, fp[f].x, i) * lagrange(p1, fp[f].y, j);
      if (nDims == 3) v = v * lagrange(p1, fp[f].z, k);
      op.ext[(size_t)f * nS + s] = v;
    }

  // opp_grad_spts[d] (operators.cpp:596-655)
  for (int d = 0; d < nDims; d++) {
    op.grad[d].assign((size_t)nS * nS, 0.0);
    for (int g = 0; g < nS; g++) {
      int gi, gj, gk;
      ijk(g, gi, gj, gk);
      for (int b = 0; b < nS; b++) {
        int bi, bj, bk;
        ijk(b, bi, bj, bk);
        double v;
        if (nDims == 2) {
          if (d == 0)
            v = dlagrange(p1, p1[gi], bi) * lagrange(p1, p1[gj], bj);
          else
            v = dlagrange(p1, p1[gj], bj) * lagrange(p1, p1[gi], bi);
        } else {
          if (d == 0)
            v = dlagrange(p1, p1[gi], bi) * lagrange(p1, p1[gj], bj) * lagrange(p1, p1[gk], bk);
          else if (d == 1)
            v = dlagrange(p1, p1[gj], bj) * lagrange(p1, p1[gi], bi) * lagrange(p1, p1[gk], bk);
          else
            v = dlagrange(p1, p1[gk], bk) * lagrange(p1, p1[gi], bi) * lagrange(p1, p1[gj], bj);
        }
        op.grad[d][(size_t)g * nS + b] = v;
      }
    }
  }

  // reference normals and opp_extrapolateFn (operators.cpp:715-797)
  op.tNorm.assign((size_t)nF * nDims, 0.0);
  for (int d = 0; d < nDims; d++) op.extFn[d].assign((size_t)nF * nS, 0.0);
  for (int f = 0; f < nF; f++) {
    double t[3];
    face_normal(nDims, f / nPF, t);
    for (int d = 0; d < nDims; d++) {
      op.tNorm[(size_t)f * nDims + d] = t[d];
      for (int s = 0; s < nS; s++) op.extFn[d][(size_t)f * nS + s] = op.ext[(size_t)f * nS + s] * t[d];
    }
  }

  // opp_correction via divVCJH (operators.cpp:800-824, 1449-1506)
  double eta = vcjh == 0 ? 0.0 : compute_eta(vcjh, order);
  op.corr.assign((size_t)nS * nF, 0.0);
  for (int s = 0; s < nS; s++) {
    const Pt &L = sp[s];
    for (int f = 0; f < nF; f++) {
      double v = 0.0;
      if (nDims == 2) {
        int i = f / n, j = f - n * i;
        if (i == 0)
          v = -lagrange(p1, L.x, j) * dvcjh_1d(L.y, 0, order, eta);
        else if (i == 1)
          v = lagrange(p1, L.y, j) * dvcjh_1d(L.x, 1, order, eta);
        else if (i == 2)
          v = lagrange(p1, L.x, order - j) * dvcjh_1d(L.y, 1, order, eta);
        else
          v = -lagrange(p1, L.y, order - j) * dvcjh_1d(L.x, 0, order, eta);
      } else {
        int P12 = n * n;
        int fc = f / P12;
        int j = (f - P12 * fc) / n;
        int i = f - P12 * fc - n * j;
        if (fc == 0)
          v = lagrange(p1, L.x, i) * lagrange(p1, L.y, j) * -dvcjh_1d(L.z, 0, order, eta);
        else if (fc == 1)
          v = lagrange(p1, L.x, order - i) * lagrange(p1, L.y, j) * dvcjh_1d(L.z, 1, order, eta);
        else if (fc == 2)
          v = lagrange(p1, L.y, i) * lagrange(p1, L.z, j) * -dvcjh_1d(L.x, 0, order, eta);
        else if (fc == 3)
          v = lagrange(p1, L.y, order - i) * lagrange(p1, L.z, j) * dvcjh_1d(L.x, 1, order, eta);
        else if (fc == 4)
          v = lagrange(p1, L.x, order - i) * lagrange(p1, L.z, j) * -dvcjh_1d(L.y, 0, order, eta);
        else
          v = lagrange(p1, L.x, i) * lagrange(p1, L.z, j) * dvcjh_1d(L.y, 1, order, eta);
      }
      op.corr[(size_t)s * nF + f] = v;
    }
  }

  // opp_correctU[d] = opp_correction * tNorm[d] (operators.cpp:915-1001)
  for (int d = 0; d < nDims; d++) {
    op.corrU[d].assign((size_t)nS * nF, 0.0);
    for (int f = 0; f < nF; f++)
      for (int s = 0; s < nS; s++)
        op.corrU[d][(size_t)s * nF + f] = op.corr[(size_t)s * nF + f] * op.tNorm[(size_t)f * nDims + d];
  }

  // P-multigrid prolongation / restriction (operators.cpp:1552-1634)
  int nPro1 = order + 2, nRes1 = order;
  op.nSptsPro = nDims == 2 ? nPro1 * nPro1 : nPro1 * nPro1 * nPro1;
  op.nSptsRes = nDims == 2 ? nRes1 * nRes1 : nRes1 * nRes1 * nRes1;
  auto proPts = pts1d(ptsType, order + 1);
  op.prolong.assign((size_t)op.nSptsPro * nS, 0.0);
  for (int s = 0; s < nS; s++) {
    int i, j, k;
    ijk(s, i, j, k);
    for (int q = 0; q < op.nSptsPro; q++) {
      double v;
      if (nDims == 2) {
        v = lagrange(p1, proPts[q % nPro1], i) * lagrange(p1, proPts[q / nPro1], j);
      } else {
        int kq = q / (nPro1 * nPro1), jq = (q - nPro1 * nPro1 * kq) / nPro1,
            iq = q - nPro1 * jq - nPro1 * nPro1 * kq;
        v = lagrange(p1, proPts[iq], i) * lagrange(p1, proPts[jq], j) * lagrange(p1, proPts[kq], k);
      }
      op.prolong[(size_t)q * nS + s] = v;
    }
  }
  if (order > 0) {
    auto resPts = pts1d(ptsType, order - 1);
    op.restrict_.assign((size_t)op.nSptsRes * nS, 0.0);
    for (int s = 0; s < nS; s++) {
      int i, j, k;
      ijk(s, i, j, k);
      for (int q = 0; q < op.nSptsRes; q++) {
        double v;
        if (nDims == 2) {
          v = lagrange(p1, resPts[q % nRes1], i) * lagrange(p1, resPts[q / nRes1], j);
        } else {
          int kq = q / (nRes1 * nRes1), jq = (q - nRes1 * nRes1 * kq) / nRes1,
              iq = q - nRes1 * jq - nRes1 * nRes1 * kq;
          v = lagrange(p1, resPts[iq], i) * lagrange(p1, resPts[jq], j) * lagrange(p1, resPts[kq], k);
        }
        op.restrict_[(size_t)q * nS + s] = v;
      }
    }
  } else {
    op.nSptsRes = 0;
  }
}

}  // namespace fr
