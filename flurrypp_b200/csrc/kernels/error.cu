// Error integrals against the exact solution of the test cases (testCase 1).
//
// solver::integrateError (src/solver.cpp:1945-2028) with the point-wise error
// of calcError (src/funcs.cpp:1318-1476): for errorNorm 0 the state itself is
// integrated with the solution-point quadrature; for errorNorm 1 and 2 the
// state and detJ are interpolated to a (quadOrder+1)^d Gauss-Legendre set and
// |error| or error^2 is integrated (2: square root of the sum).  The exact
// fields are the deck's: icType 0 the entropy error of the free stream,
// icType 1 the Kui vortex advected with (1, 1), icType 2 the Liang-Miyaji
// vortex advected along vortexAngle, both wrapped periodically.
//
// One CTA per element sums its evaluation points (tree reduction in shared
// memory); one CTA then sums the elements in element order.
#include <cuda_runtime.h>

#include "launch.cuh"
#include "stage.hpp"

namespace frk {

namespace {

constexpr int kThreads = 128;
constexpr int kMaxF = 5;

__device__ void exact_error(const ErrorArgs &a, const double *U, const double *pos, double t, double *err) {
  const int nd = a.nDims, nF = a.nF;
  for (int k = 0; k < nF; k++) err[k] = a.testCase == 0 ? U[k] : 0.0;
  if (a.testCase != 0) {
    const double gamma = a.gamma, pi = a.pi;
    if (a.icType == 0) {  // free stream: entropy error
      const double pfs = a.pIC, rhofsg = pow(a.rhoIC, gamma);
      const double rho = U[0], u = U[1] / rho, v = U[2] / rho, w = nd == 2 ? 0.0 : U[3] / rho;
      const double p = (gamma - 1.) * (U[nd + 1] - .5 * rho * (u * u + v * v + w * w));
      err[0] = p * rhofsg / (pow(rho, gamma) * pfs) - 1.;
    } else {
      double rho, vx, vy, p;
      const double xmin = a.xmin, xmax = a.xmax, ymin = a.ymin, ymax = a.ymax;
      if (a.icType == 1) {  // Kui vortex, eps 5, advected with (1, 1)
        const double eps = 5.0;
        double x = fmod((pos[0] - t), (xmax - xmin));
        double y = fmod((pos[1] - t), (ymax - ymin));
        if (x > xmax) x -= (xmax - xmin);
        if (y > ymax) y -= (ymax - ymin);
        if (x < xmin) x += (xmax - xmin);
        if (y < ymin) y += (ymax - ymin);
        const double f = 1.0 - (x * x + y * y);
        rho = fmax(pow(1. - eps * eps * (gamma - 1.) / (8. * gamma * pi * pi) * exp(f), 1.0 / (gamma - 1.0)), 1e-10);
        vx = 1. - eps * y / (2. * pi) * exp(f / 2.);
        vy = 1. + eps * x / (2. * pi) * exp(f / 2.);
        p = pow(rho, gamma);
      } else {  // Liang-Miyaji vortex
        const double eps = 1.0, rc = 1.0, Minf = .3, Uinf = 1, rhoInf = 1, theta = a.vortexAngle;
        const double Pinf = pow(Minf, -2) / gamma;
        const double eM = (eps * Minf) * (eps * Minf);
        const double advX = Uinf * cos(theta) * t, advY = Uinf * sin(theta) * t;
        double x = (fmod((pos[0] - advX), (xmax - xmin)));
        double y = (fmod((pos[1] - advY), (ymax - ymin)));
        if (x > xmax) x -= (xmax - xmin);
        if (x < xmin) x += (xmax - xmin);
        if (y > ymax) y -= (ymax - ymin);
        if (y < ymin) y += (ymax - ymin);
        const double f = -(x * x + y * y) / (rc * rc);
        vx = Uinf * (cos(theta) - y * eps / rc * exp(f / 2.));
        vy = Uinf * (sin(theta) + x * eps / rc * exp(f / 2.));
        rho = rhoInf * pow(1. - (gamma - 1.) / 2. * eM * exp(f), gamma / (gamma - 1.0));
        p = Pinf * pow(1. - (gamma - 1.) / 2. * eM * exp(f), gamma / (gamma - 1.0));
      }
      double ex[kMaxF];
      ex[0] = rho;
      ex[1] = rho * vx;
      ex[2] = rho * vy;
      if (nd == 3) ex[3] = 0.;
      ex[nd + 1] = p / (gamma - 1) + (0.5 * rho * (vx * vx + vy * vy));
      for (int k = 0; k < nF; k++) err[k] = U[k] - ex[k];
    }
  }
  if (a.errorNorm == 1)
    for (int k = 0; k < nF; k++) err[k] = fabs(err[k]);
  else if (a.errorNorm == 2)
    for (int k = 0; k < nF; k++) err[k] *= err[k];
}

__global__ void __launch_bounds__(kThreads) k_error_elements(ErrorArgs a) {
  pdl_wait();
  pdl_trigger();
  __shared__ double sh[kThreads][2 * kMaxF];
  const int e = blockIdx.x, nS = a.nS, nF = a.nF, E = a.E, nd = a.nDims;
  const double t = *a.time;
  double accE[kMaxF], accU[kMaxF];
  for (int k = 0; k < kMaxF; k++) accE[k] = accU[k] = 0.0;
  for (int q = threadIdx.x; q < a.nQ; q += kThreads) {
    const double *op = a.opQ + (size_t)q * nS;
    double Uq[kMaxF] = {0, 0, 0, 0, 0}, dJ = 0.0, pos[3] = {0, 0, 0};
    for (int s = 0; s < nS; s++) {
      const double w = op[s];
      const double *u = a.U + ((size_t)s * E + e) * nF;
      for (int k = 0; k < nF; k++) Uq[k] += w * u[k];
      dJ += w * a.detJ[(size_t)s * E + e];
    }
    const double *N = a.shapeQ + (size_t)q * a.nNodes;
    for (int n = 0; n < a.nNodes; n++) {
      const double *x = a.xv + (size_t)a.c2v[(size_t)e * a.nNodes + n] * nd;
      for (int d = 0; d < nd; d++) pos[d] += N[n] * x[d];
    }
    double err[kMaxF];
    exact_error(a, Uq, pos, t, err);
    const double wq = a.wQ[q];
    for (int k = 0; k < nF; k++) {
      accE[k] += err[k] * wq * dJ;
      accU[k] += Uq[k] * wq * dJ;
    }
  }
  for (int k = 0; k < nF; k++) {
    sh[threadIdx.x][k] = accE[k];
    sh[threadIdx.x][kMaxF + k] = accU[k];
  }
  __syncthreads();
  for (int half = kThreads / 2; half > 0; half >>= 1) {
    if ((int)threadIdx.x < half)
      for (int k = 0; k < 2 * kMaxF; k++) sh[threadIdx.x][k] += sh[threadIdx.x + half][k];
    __syncthreads();
  }
  if (threadIdx.x < (unsigned)nF) {
    a.elemErr[(size_t)e * nF + threadIdx.x] = sh[0][threadIdx.x];
    a.elemU[(size_t)e * nF + threadIdx.x] = sh[0][kMaxF + threadIdx.x];
  }
}

// Sums the per-element integrals; errorNorm 0 reports |int(U - exact) - int U|
// and 2 the square root (src/solver.cpp:1960-1966, 2024-2025).
__global__ void __launch_bounds__(kThreads) k_error_total(ErrorArgs a, double *out) {
  pdl_wait();
  pdl_trigger();
  __shared__ double sh[kThreads][2 * kMaxF];
  const int nF = a.nF;
  double accE[kMaxF], accU[kMaxF];
  for (int k = 0; k < kMaxF; k++) accE[k] = accU[k] = 0.0;
  for (int e = threadIdx.x; e < a.E; e += kThreads)
    for (int k = 0; k < nF; k++) {
      accE[k] += a.elemErr[(size_t)e * nF + k];
      accU[k] += a.elemU[(size_t)e * nF + k];
    }
  for (int k = 0; k < nF; k++) {
    sh[threadIdx.x][k] = accE[k];
    sh[threadIdx.x][kMaxF + k] = accU[k];
  }
  __syncthreads();
  for (int half = kThreads / 2; half > 0; half >>= 1) {
    if ((int)threadIdx.x < half)
      for (int k = 0; k < 2 * kMaxF; k++) sh[threadIdx.x][k] += sh[threadIdx.x + half][k];
    __syncthreads();
  }
  if (threadIdx.x < (unsigned)nF) {
    double v = a.errorNorm == 0 ? fabs(sh[0][threadIdx.x] - sh[0][kMaxF + threadIdx.x]) : sh[0][threadIdx.x];
    if (a.errorNorm == 2) v = sqrt(fabs(v));
    out[threadIdx.x] = v;
  }
}

}  // namespace

void launch_error_integral(const ErrorArgs &a, double *out, cudaStream_t st) {
  if (a.E <= 0) return;
  launch_k(k_error_elements, a.E, kThreads, 0, st, a);
  launch_k(k_error_total, 1, kThreads, 0, st, a, out);
}

}  // namespace frk
