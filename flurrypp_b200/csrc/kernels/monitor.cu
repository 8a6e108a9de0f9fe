// Boundary monitors: forces on walls and the mass flux through inflow and
// outflow boundaries.
//
// boundFace::computeWallForce (src/boundFace.cpp:412-458): on slip,
// adiabatic and isothermal walls, the pressure force sum p n dA w and, for
// viscous runs, the viscous force -tau . n dA w (viscousStressTensor,
// src/flux.cpp:212-340); boundFace::computeMassFlux (src/boundFace.cpp:
// 460-496): on characteristic, supersonic and subsonic inflow/outflow faces,
// the face's common flux Fn dA w (errorNorm 0), |Fn dA| w n_x (1) or
// (Fn dA)^2 w n_x (2).  w is the Gauss weight of the flux point within its
// face.  Both read the face data of the last residual evaluation: the left
// traces U_fpts, the common flux Fn_fpts = Fn dA and, viscous, the corrected
// gradients at the flux points.
//
// One thread per boundary face point writes its contributions; one CTA then
// sums them in point order.
#include <cuda_runtime.h>

#include <type_traits>

#include "launch.cuh"
#include "stage.hpp"

namespace frk {

namespace {

constexpr int kThreads = 256;
constexpr int kParts = 6 + 5;  // force (pressure xyz, viscous xyz), mass flux per field

template <int ND, typename R>
__global__ void __launch_bounds__(kThreads) k_boundary_parts(MonitorArgsT<R> a) {
  pdl_wait();
  pdl_trigger();
  constexpr int NF = ND + 2;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = a.nI + t;
  if (i >= a.n) return;
  double *part = a.part + (size_t)t * kParts;
  for (int k = 0; k < kParts; k++) part[k] = 0.0;
  const int bc = -a.slotR[i] - 2, sL = a.slotL[i];
  const int j = (sL / a.E) % a.nPF;  // flux point within its face
  const double w = a.wSurf[j];
  const double dA = (double)a.dAL[i];
  double n[ND];
  for (int d = 0; d < ND; d++) n[d] = (double)a.nrm[(size_t)i * ND + d];
  const bool wall = bc == BC_SLIP_WALL || bc == BC_ADI_NOSLIP || bc == BC_ISO_NOSLIP;
  const bool through = bc == BC_CHAR || bc == BC_SUP_IN || bc == BC_SUP_OUT || bc == BC_SUB_IN || bc == BC_SUB_OUT;
  if (wall) {
    double U[NF];
    for (int k = 0; k < NF; k++) U[k] = (double)a.Uf[(size_t)sL * NF + k];
    const double rho = U[0];
    double vMagSq = 0;
    for (int d = 0; d < ND; d++) vMagSq += U[d + 1] * U[d + 1] / (rho * rho);
    const double p = (a.ph.gamma - 1) * (U[ND + 1] - 0.5 * rho * vMagSq);
    for (int d = 0; d < ND; d++) part[d] += p * n[d] * dA * w;
    if (a.dUf) {
      double g[ND][NF];
      for (int d = 0; d < ND; d++)
        for (int k = 0; k < NF; k++) g[d][k] = (double)a.dUf[d * a.fStride + (long long)sL * NF + k];
      // viscousStressTensor (src/flux.cpp:212-340), with the reference's
      // 3-D off-diagonal entries when the 3-D flux quirk is on
      const double u = U[1] / rho, v = U[2] / rho, ww = ND == 3 ? U[3] / rho : 0.0;
      double e = U[ND + 1] / rho - 0.5 * (u * u + v * v);
      if (ND == 3) e -= 0.5 * (ww * ww);
      double mu = a.ph.mu_inf;
      if (!a.ph.fixVis) {
        const double rt = (a.ph.gamma - 1.0) * e / a.ph.rt_inf;
        mu *= pow(rt, 1.5) * (1. + a.ph.c_sth) / (rt + a.ph.c_sth);
      }
      const double du_dx = (g[0][1] - g[0][0] * u) / rho, du_dy = (g[1][1] - g[1][0] * u) / rho;
      const double dv_dx = (g[0][2] - g[0][0] * v) / rho, dv_dy = (g[1][2] - g[1][0] * v) / rho;
      double du_dz = 0, dv_dz = 0, dw_dx = 0, dw_dy = 0, dw_dz = 0;
      if (ND == 3) {
        du_dz = (g[ND - 1][1] - g[ND - 1][0] * u) / rho;
        dv_dz = (g[ND - 1][2] - g[ND - 1][0] * v) / rho;
        dw_dx = (g[0][ND == 3 ? 3 : 0] - g[0][0] * ww) / rho;
        dw_dy = (g[1][ND == 3 ? 3 : 0] - g[1][0] * ww) / rho;
        dw_dz = (g[ND - 1][ND == 3 ? 3 : 0] - g[ND - 1][0] * ww) / rho;
      }
      const double diag = (du_dx + dv_dy + dw_dz) / 3.0;
      double tau[3][3];
      tau[0][0] = 2.0 * mu * (du_dx - diag);
      tau[1][1] = 2.0 * mu * (dv_dy - diag);
      tau[0][1] = tau[1][0] = mu * (du_dy + dv_dx);
      if (ND == 3) {
        const bool quirk = a.ph.viscFluxQuirk;
        tau[0][2] = tau[2][0] = mu * (du_dz + (quirk ? dv_dx : dw_dx));
        tau[1][2] = tau[2][1] = mu * ((quirk ? du_dz : dv_dz) + (quirk ? dv_dy : dw_dy));
        tau[2][2] = 2.0 * mu * (dw_dz - diag);
      }
      for (int d1 = 0; d1 < ND; d1++)
        for (int d2 = 0; d2 < ND; d2++) part[3 + d1] -= tau[d1][d2] * n[d2] * dA * w;
    }
  } else if (through) {
    for (int k = 0; k < NF; k++) {
      const double f = (double)a.Fn[(size_t)sL * NF + k];  // Fn dA of the left side
      if (a.errorNorm == 0)
        part[6 + k] = f * w;
      else if (a.errorNorm == 1)
        part[6 + k] = fabs(f) * w * n[0];
      else
        part[6 + k] = f * f * w * n[0];
    }
  }
}

__global__ void __launch_bounds__(kThreads) k_boundary_total(int nB, const double *__restrict__ part,
                                                            double *__restrict__ out) {
  pdl_wait();
  pdl_trigger();
  __shared__ double sh[kThreads][kParts];
  double acc[kParts];
  for (int k = 0; k < kParts; k++) acc[k] = 0.0;
  for (int t = threadIdx.x; t < nB; t += kThreads)
    for (int k = 0; k < kParts; k++) acc[k] += part[(size_t)t * kParts + k];
  for (int k = 0; k < kParts; k++) sh[threadIdx.x][k] = acc[k];
  __syncthreads();
  for (int half = kThreads / 2; half > 0; half >>= 1) {
    if ((int)threadIdx.x < half)
      for (int k = 0; k < kParts; k++) sh[threadIdx.x][k] += sh[threadIdx.x + half][k];
    __syncthreads();
  }
  if (threadIdx.x < kParts) out[threadIdx.x] = sh[0][threadIdx.x];
}

}  // namespace

template <typename R>
void launch_boundary_monitors(int nDims, const MonitorArgsT<R> &a, double *out, cudaStream_t st) {
  const int nB = a.n - a.nI;
  if (nB <= 0) {
    cudaMemsetAsync(out, 0, kParts * sizeof(double), st);
    return;
  }
  const unsigned g = (unsigned)((nB + kThreads - 1) / kThreads);
  if (nDims == 2)
    launch_k(k_boundary_parts<2, R>, g, kThreads, 0, st, a);
  else
    launch_k(k_boundary_parts<3, R>, g, kThreads, 0, st, a);
  launch_k(k_boundary_total, 1, kThreads, 0, st, nB, (const double *)a.part, out);
}

template void launch_boundary_monitors<double>(int, const MonitorArgsT<double> &, double *, cudaStream_t);
template void launch_boundary_monitors<float>(int, const MonitorArgsT<float> &, double *, cudaStream_t);

}  // namespace frk
