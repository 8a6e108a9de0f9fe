// Moving meshes (deck option "motion"), FP64 plain form.
//
// The reference moves the mesh vertices at every RK stage by an analytic
// law (geo::moveMesh, src/geo.cpp:2730-2830), rebuilds the solution- and
// flux-point positions, grid velocities and metric terms from the moved
// vertices (solver::moveMesh / updatePosSptsFpts / updateGridVSptsFpts /
// calcTransforms, src/solver.cpp:1168-1246, 1316-1394, 1587-1694), and
// evaluates the residual in the non-conservative chain-rule form of Liang,
// Miyaji and Zhang (AIAA 2013-0998): the physical flux and the solution are
// differentiated in reference space and combined with the adjugate of the
// space-time Jacobian (solver::calcGradF_spts / transformGradF_spts,
// src/solver.cpp:836-904), the interface correction uses the extrapolated
// physical normal flux (solver::extrapolateNormalFlux, src/solver.cpp:956-995).
//
// Everything here runs on the device from device-resident time and dt, so
// the whole moving-mesh step is graph-capturable.  The kernels are simple
// one-thread-per-point passes over global memory: moving meshes are an
// option of the path, not its throughput case.
#include <cuda_runtime.h>

#include "fr_physics.cuh"
#include "launch.cuh"
#include "stage.hpp"

namespace frk {

namespace {

constexpr double kPi = 3.141592653589793238462643383279502884;

// Vertex positions and velocities at rkTime = time + dt * rkVal.
__global__ void k_move_vertices(MotionArgs m, double rkVal) {
  pdl_wait();
  pdl_trigger();
  const int iv = blockIdx.x * blockDim.x + threadIdx.x;
  if (iv >= m.nVerts) return;
  const int nd = m.nDims;
  const double t = *m.time + *m.dt * rkVal;
  const double *x0 = m.xv0 + (size_t)iv * nd;
  double *x = m.xv + (size_t)iv * nd, *g = m.gv + (size_t)iv * nd;
  const double pi = kPi;
  switch (m.type) {
    case 1: {  // perturbation test case (Kui, AIAA-2010-5031-661)
      const double DX = 0.5 * m.DX, DY = 0.5 * m.DY;
      const double a = sin(pi * x0[0] / DX) * sin(pi * x0[1] / DY);
      x[0] = x0[0] + a * sin(2 * pi * t / 10.);
      x[1] = x0[1] + a * sin(2 * pi * t / 10.);
      g[0] = 2. * pi / 10. * a * cos(2 * pi * t / 10.);
      g[1] = 2. * pi / 10. * a * cos(2 * pi * t / 10.);
      break;
    }
    case 2:
    case 3: {  // Liang-Miyaji deformation on a domain of width 5
      const double t0 = 10. * sqrt(5.), w = 5.;
      if (nd == 2) {
        const double a = sin(pi * x0[0] / w) * sin(pi * x0[1] / w);
        x[0] = x0[0] + a * sin(4 * pi * t / t0);
        x[1] = x0[1] + a * sin(8 * pi * t / t0);
        g[0] = 4. * pi / t0 * a * cos(4 * pi * t / t0);
        g[1] = 8. * pi / t0 * a * cos(8 * pi * t / t0);
      } else if (m.type == 2) {
        const double a = sin(pi * x0[0] / w) * sin(pi * x0[1] / w) * sin(pi * x0[2] / w);
        x[0] = x0[0] + a * sin(4 * pi * t / t0);
        x[1] = x0[1] + a * sin(8 * pi * t / t0);
        x[2] = x0[2] + a * sin(4 * pi * t / t0);
        g[0] = 4. * pi / t0 * a * cos(4 * pi * t / t0);
        g[1] = 8. * pi / t0 * a * cos(8 * pi * t / t0);
        g[2] = 4. * pi / t0 * a * cos(4 * pi * t / t0);
      }
      break;
    }
    case 4: {  // rigid oscillation
      x[0] = x0[0] + m.Ax * sin(2. * pi * m.Fx * t);
      x[1] = x0[1] + m.Ay * (1 - cos(2. * pi * m.Fy * t));
      g[0] = 2. * pi * m.Fx * m.Ax * cos(2. * pi * m.Fx * t);
      g[1] = 2. * pi * m.Fy * m.Ay * sin(2. * pi * m.Fy * t);
      break;
    }
    case 5: {  // radial expansion / contraction (3-D)
      const double *r0 = m.rv0 + (size_t)iv * 3;
      const double r = r0[0] + m.Ar * (1. - cos(2. * pi * m.Fr * t));
      const double rdot = 2. * pi * m.Ar * m.Fr * sin(2. * pi * m.Fr * t);
      const double th = r0[1], ps = r0[2];
      x[0] = r * sin(ps) * cos(th);
      x[1] = r * sin(ps) * sin(th);
      x[2] = r * cos(ps);
      g[0] = rdot * sin(ps) * cos(th);
      g[1] = rdot * sin(ps) * sin(th);
      g[2] = rdot * cos(ps);
      break;
    }
  }
}

// Positions are not needed by the residual; grid velocities at every point,
// and (unless the motion is a rigid translation) the Jacobian, its adjugate,
// detJ, and at the flux points the unit normal and dA.  Points [0, nS) are
// solution points, [nS, nS + nFp) flux points.
template <int ND>
__global__ void k_motion_geometry(MotionArgs m, int transforms) {
  pdl_wait();
  pdl_trigger();
  const int nS = m.nS, nFp = m.nFp, E = m.E, nN = m.nNodes;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)(nS + nFp) * E) return;
  const int e = (int)(t % E), p = (int)(t / E);
  const int *cv = m.c2v + (size_t)e * nN;
  const double *N = m.shape + (size_t)p * nN;
  const double *dN = m.dshape + (size_t)p * nN * ND;
  double J[ND][ND], gV[ND];
#pragma unroll
  for (int a = 0; a < ND; a++) {
    gV[a] = 0.0;
#pragma unroll
    for (int b = 0; b < ND; b++) J[a][b] = 0.0;
  }
  for (int n = 0; n < nN; n++) {
    const double *x = m.xv + (size_t)cv[n] * ND, *g = m.gv + (size_t)cv[n] * ND;
#pragma unroll
    for (int d = 0; d < ND; d++) {
      gV[d] += N[n] * g[d];
#pragma unroll
      for (int r = 0; r < ND; r++) J[r][d] += dN[n * ND + r] * x[d];
    }
  }
  if (p < nS) {
#pragma unroll
    for (int d = 0; d < ND; d++) m.gVs[((size_t)p * E + e) * ND + d] = gV[d];
  } else {
#pragma unroll
    for (int d = 0; d < ND; d++) m.gVf[((size_t)(p - nS) * E + e) * ND + d] = gV[d];
  }
  if (!transforms) return;
  // J[r][d] = d x_d / d xi_r; A = adjugate (JGinv), src/solver.cpp:1612-1636
  double det, A[ND][ND];
  if constexpr (ND == 2) {
    det = J[0][0] * J[1][1] - J[0][1] * J[1][0];
    A[0][0] = J[1][1];
    A[0][1] = -J[1][0];
    A[1][0] = -J[0][1];
    A[1][1] = J[0][0];
  } else {
    const double xr = J[0][0], xs = J[1][0], xt = J[2][0];
    const double yr = J[0][1], ys = J[1][1], yt = J[2][1];
    const double zr = J[0][2], zs = J[1][2], zt = J[2][2];
    det = xr * (ys * zt - yt * zs) - xs * (yr * zt - yt * zr) + xt * (yr * zs - ys * zr);
    A[0][0] = ys * zt - yt * zs;
    A[0][1] = xt * zs - xs * zt;
    A[0][2] = xs * yt - xt * ys;
    A[1][0] = yt * zr - yr * zt;
    A[1][1] = xr * zt - xt * zr;
    A[1][2] = xt * yr - xr * yt;
    A[2][0] = yr * zs - ys * zr;
    A[2][1] = xs * zr - xr * zs;
    A[2][2] = xr * ys - xs * yr;
  }
  if (p < nS) {
    if (det < 0 && m.err) atomicOr(m.err, 2u);  // the reference stops: "Negative Jacobian"
    m.detJ[(size_t)p * E + e] = det;
#pragma unroll
    for (int r = 0; r < ND; r++)
#pragma unroll
      for (int d = 0; d < ND; d++) {
        m.Jac[(((size_t)r * nS + p) * E + e) * ND + d] = J[r][d];
        m.JGinv[(((size_t)r * nS + p) * E + e) * ND + d] = A[r][d];
      }
    return;
  }
  const int f = p - nS;
  const double *tn = m.tNorm + (size_t)f * ND;
  double nv[ND], dA = 0.0;
#pragma unroll
  for (int d1 = 0; d1 < ND; d1++) {
    nv[d1] = 0.0;
#pragma unroll
    for (int d2 = 0; d2 < ND; d2++) nv[d1] += A[d2][d1] * tn[d2];
  }
#pragma unroll
  for (int d = 0; d < ND; d++) dA += nv[d] * nv[d];
  dA = sqrt(dA);
  if (fabs(dA) < 1e-10) {
    dA = 0.0;
#pragma unroll
    for (int d = 0; d < ND; d++) nv[d] = 0.0;
  } else {
#pragma unroll
    for (int d = 0; d < ND; d++) nv[d] /= dA;
  }
  m.dA[(size_t)f * E + e] = dA;
#pragma unroll
  for (int d = 0; d < ND; d++) m.norm[((size_t)f * E + e) * ND + d] = nv[d];
}

// The face table's copies of the normals and dA from the moved metrics.
__global__ void k_face_refresh(int n, int nDims, const int *__restrict__ slotL, const int *__restrict__ slotR,
                               const double *__restrict__ norm, const double *__restrict__ dA, double *nrm,
                               double *dAL, double *dAR) {
  pdl_wait();
  pdl_trigger();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int sL = slotL[i], sR = slotR[i];
  for (int d = 0; d < nDims; d++) nrm[(size_t)i * nDims + d] = norm[(size_t)sL * nDims + d];
  dAL[i] = dA[sL];
  dAR[i] = sR >= 0 ? dA[sR] : 0.0;
}

// Rusanov common flux at every face point with the left element's grid
// velocity (face.cpp:120-208, 314-374; boundFace.cpp:65-314).
template <int ND>
__global__ void __launch_bounds__(256) k_faces_motion(FaceTableT<double> ft, const double *__restrict__ Uf,
                                                      double *__restrict__ Fn, double *__restrict__ waveSp,
                                                      const double *__restrict__ gVf, Phys ph) {
  pdl_wait();
  pdl_trigger();
  constexpr int NF = ND + 2;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ft.n) return;
  const int sL = ft.slotL[i], sR = ft.slotR[i];
  double UL[NF], UR[NF], nv[ND], vG[ND], F[NF];
  for (int k = 0; k < NF; k++) UL[k] = Uf[(size_t)sL * NF + k];
  double vgn = 0.0;
  for (int d = 0; d < ND; d++) {
    nv[d] = ft.nrm[(size_t)i * ND + d];
    vG[d] = gVf[(size_t)sL * ND + d];
    vgn += nv[d] * vG[d];
  }
  if (sR >= 0) {
    for (int k = 0; k < NF; k++) UR[k] = Uf[(size_t)sR * NF + k];
  } else {
    boundary_state<ND, double>(-sR - 2, UL, nv, ph, UR, vG);
  }
  const double ws = rusanov<ND, double>(UL, UR, nv, ph.gamma, F, vgn);
  if (waveSp) waveSp[sL] = ws;
  const double aL = ft.dAL[i];
  for (int k = 0; k < NF; k++) Fn[(size_t)sL * NF + k] = F[k] * aL;
  if (sR >= 0) {
    const double aR = ft.dAR[i];
    for (int k = 0; k < NF; k++) Fn[(size_t)sR * NF + k] = -F[k] * aR;
  }
}

// Wave speeds from U_fpts relative to the grid (ele::calcWaveSpFpts,
// src/ele.cpp:1076-1125, motion branch).
template <int ND>
__global__ void k_wavesp_motion(int nFp, int E, const double *__restrict__ Uf, const double *__restrict__ norm,
                                const double *__restrict__ gVf, double gamma, double *__restrict__ waveSp) {
  pdl_wait();
  pdl_trigger();
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)nFp * E) return;
  const double *u = Uf + t * (ND + 2);
  const double *n = norm + t * ND, *g = gVf + t * ND;
  const double rho = u[0];
  const double vx = u[1] / rho, vy = u[2] / rho, vz = ND == 3 ? u[3] / rho : 0.0;
  const double rhoVSq = rho * (vx * vx + vy * vy + vz * vz);
  const double p = (gamma - 1) * (u[ND + 1] - 0.5 * rhoVSq);
  double vN = vx * n[0] + vy * n[1];
  if (ND == 3) vN += vz * n[ND - 1];
  double vgN = g[0] * n[0] + g[1] * n[1];
  if (ND == 3) vgN += g[ND - 1] * n[ND - 1];
  const double csq = fmax(gamma * p / rho, 0.0);
  waveSp[t] = fabs(vN - vgN) + sqrt(csq);
}

// Physical inviscid flux at the solution points, [d][spt][ele][field].
template <int ND>
__global__ void k_motion_flux(int nS, int E, const double *__restrict__ U, double gamma, double *__restrict__ F) {
  pdl_wait();
  pdl_trigger();
  constexpr int NF = ND + 2;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)nS * E) return;
  double f[ND][NF];
  inviscid_flux<ND, double>(U + t * NF, f, gamma);
  const size_t plane = (size_t)nS * E * NF;
  for (int d = 0; d < ND; d++)
    for (int k = 0; k < NF; k++) F[d * plane + t * NF + k] = f[d][k];
}

// 3x3 determinant by expansion along the first column.
__device__ __forceinline__ double det3(const double m[3][3]) {
  return m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]) - m[1][0] * (m[0][1] * m[2][2] - m[0][2] * m[2][1]) +
         m[2][0] * (m[0][1] * m[1][2] - m[0][2] * m[1][1]);
}

// Flux divergence by the chain rule: reference-space gradients of U and of
// each physical flux component, combined with the adjugate of the
// space-time Jacobian [[dx/dxi, v_grid], [0, 1]].
template <int ND>
__global__ void k_motion_divergence(MotionArgs m, const double *__restrict__ U, const double *__restrict__ F,
                                    double *__restrict__ divF) {
  pdl_wait();
  pdl_trigger();
  constexpr int NF = ND + 2;
  const int nS = m.nS, E = m.E;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)nS * E) return;
  const int e = (int)(t % E), s = (int)(t / E);
  const size_t plane = (size_t)nS * E * NF;
  // dU[d][k] = sum_j grad_d(s, j) U(j); dF[d2][d1][k] = sum_j grad_d2(s, j) F_d1(j)
  double dU[ND][NF], dF[ND][ND][NF];
  for (int d2 = 0; d2 < ND; d2++) {
    const double *G = m.opGrad + ((size_t)d2 * nS + s) * nS;
    for (int k = 0; k < NF; k++) {
      dU[d2][k] = 0.0;
      for (int d1 = 0; d1 < ND; d1++) dF[d2][d1][k] = 0.0;
    }
    for (int j = 0; j < nS; j++) {
      const double g = G[j];
      if (g == 0.0) continue;  // structural zeros of the tensor-product operator
      const double *u = U + ((size_t)j * E + e) * NF;
      for (int k = 0; k < NF; k++) dU[d2][k] += g * u[k];
      for (int d1 = 0; d1 < ND; d1++) {
        const double *f = F + d1 * plane + ((size_t)j * E + e) * NF;
        for (int k = 0; k < NF; k++) dF[d2][d1][k] += g * f[k];
      }
    }
  }
  double J[ND][ND], gV[ND];  // J[dim][comp] = d x_comp / d xi_dim
  for (int a = 0; a < ND; a++) {
    gV[a] = m.gVs[((size_t)s * E + e) * ND + a];
    for (int b = 0; b < ND; b++) J[a][b] = m.Jac[(((size_t)a * nS + s) * E + e) * ND + b];
  }
  double *out = divF + ((size_t)s * E + e) * NF;
  if constexpr (ND == 2) {
    // src/solver.cpp:866-878
    const double A = gV[1] * J[1][0] - gV[0] * J[1][1];
    const double B = gV[0] * J[0][1] - gV[1] * J[0][0];
    for (int k = 0; k < NF; k++) {
      const double a = dF[0][0][k] * J[1][1] - dF[0][1][k] * J[1][0] + dU[0][k] * A;
      const double b = -dF[1][0][k] * J[0][1] + dF[1][1][k] * J[0][0] + dU[1][k] * B;
      out[k] = a + b;
    }
  } else {
  // 3-D: S = adjugate of the 4x4 matrix M, M(i, j) = d x_i / d xi_j,
  // M(i, 3) = v_grid_i, M(3, :) = (0, 0, 0, 1) (src/solver.cpp:881-902)
  double M[4][4];
  for (int i = 0; i < 3; i++) {
    for (int j = 0; j < 3; j++) M[i][j] = J[j][i];
    M[i][3] = gV[i];
    M[3][i] = 0.0;
  }
  M[3][3] = 1.0;
  double S[4][4];
  for (int row = 0; row < 4; row++)
    for (int col = 0; col < 4; col++) {
      double mi[3][3];
      for (int i = 0, i0 = 0; i < 4; i++) {
        if (i == row) continue;
        for (int j = 0, j0 = 0; j < 4; j++) {
          if (j == col) continue;
          mi[i0][j0++] = M[i][j];
        }
        i0++;
      }
      S[col][row] = ((row + col) % 2 ? -1.0 : 1.0) * det3(mi);
    }
  for (int k = 0; k < NF; k++) {
    double v = 0.0;
    for (int d1 = 0; d1 < 3; d1++)
      for (int d2 = 0; d2 < 3; d2++) v += dF[d2][d1][k] * S[d2][d1];
    for (int d = 0; d < 3; d++) v += dU[d][k] * S[d][3];
    out[k] = v;
  }
  }
}

// Fn - (extrapolated physical flux) . n dA at the flux points
// (solver::extrapolateNormalFlux motion branch and correctDivFlux's first
// pass, src/solver.cpp:956-995, 1036-1044).
template <int ND>
__global__ void k_motion_normal_flux(MotionArgs m, const double *__restrict__ F, const double *__restrict__ Fn,
                                     double *__restrict__ disFn) {
  pdl_wait();
  pdl_trigger();
  constexpr int NF = ND + 2;
  const int nS = m.nS, nFp = m.nFp, E = m.E;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)nFp * E) return;
  const int e = (int)(t % E), f = (int)(t / E);
  const size_t plane = (size_t)nS * E * NF;
  const double *X = m.opExt + (size_t)f * nS;
  const double dA = m.dA[t];
  const double *n = m.norm + t * ND;
  double acc[NF];
  for (int d = 0; d < ND; d++) {
    double v[NF];
    for (int k = 0; k < NF; k++) v[k] = 0.0;
    for (int j = 0; j < nS; j++) {
      const double x = X[j];
      if (x == 0.0) continue;
      const double *q = F + d * plane + ((size_t)j * E + e) * NF;
      for (int k = 0; k < NF; k++) v[k] += x * q[k];
    }
    for (int k = 0; k < NF; k++) acc[k] = d == 0 ? v[k] * (n[0] * dA) : acc[k] + v[k] * n[d] * dA;
  }
  for (int k = 0; k < NF; k++) disFn[t * NF + k] = Fn[t * NF + k] - acc[k];
}

// divF += correction operator . (Fn - disFn) (correctDivFlux, src/solver.cpp:1046-1057).
template <int ND>
__global__ void k_motion_correct(MotionArgs m, const double *__restrict__ disFn, double *__restrict__ divF) {
  pdl_wait();
  pdl_trigger();
  constexpr int NF = ND + 2;
  const int nS = m.nS, nFp = m.nFp, E = m.E;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)nS * E) return;
  const int e = (int)(t % E), s = (int)(t / E);
  const double *C = m.opCorr + (size_t)s * nFp;
  double acc[NF];
  for (int k = 0; k < NF; k++) acc[k] = 0.0;
  for (int f = 0; f < nFp; f++) {
    const double c = C[f];
    if (c == 0.0) continue;
    const double *q = disFn + ((size_t)f * E + e) * NF;
    for (int k = 0; k < NF; k++) acc[k] += c * q[k];
  }
  double *out = divF + t * NF;
  for (int k = 0; k < NF; k++) out[k] = acc[k] + out[k];
}

// U = U0 - RKval (divF + src) / detJ dt (timeStepA, src/solver.cpp:470-500;
// src is the P-multigrid source term of a coarse level, or null).
__global__ void k_motion_step_a(long long nSE, int nF, int E, const double *__restrict__ U0,
                                const double *__restrict__ divF, const double *__restrict__ src,
                                const double *__restrict__ detJ, const double *__restrict__ dt,
                                const double *__restrict__ eleDt, double rk, double *__restrict__ U) {
  pdl_wait();
  pdl_trigger();
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nSE * nF) return;
  const long long se = t / nF;
  const double h = eleDt ? eleDt[se % E] : *dt;
  const double d = src ? divF[t] + src[t] : divF[t];
  U[t] = U0[t] - rk * d / detJ[se] * h;
}

// The final combination of a standard RK step: U = U0 (or U for a
// one-stage scheme), then U -= RKb[s] divF[s] / detJ dt for every stage in
// order, all with the metrics of the last stage (timeStepB, src/solver.cpp:344-355, 502-535).
// A coarse P-multigrid level adds its source term to every stage residual
// (src/solver.cpp:470-535 with PMG_Source).
__global__ void k_motion_step_b(long long nSE, int nF, int E, const double *__restrict__ base,
                                MotionStages st, const double *__restrict__ src, const double *__restrict__ detJ,
                                const double *__restrict__ dt, const double *__restrict__ eleDt,
                                double *__restrict__ U) {
  pdl_wait();
  pdl_trigger();
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nSE * nF) return;
  const long long se = t / nF;
  const double h = eleDt ? eleDt[se % E] : *dt;
  double u = base[t];
  for (int s = 0; s < st.n; s++) {
    const double d = src ? st.divF[s][t] + src[t] : st.divF[s][t];
    u -= st.rkb[s] * d / detJ[se] * h;
  }
  U[t] = u;
}

unsigned blocks_for(long long n, int threads) { return (unsigned)((n + threads - 1) / threads); }

}  // namespace

void launch_move_vertices(const MotionArgs &m, double rkVal, cudaStream_t st) {
  if (m.nVerts > 0) launch_k(k_move_vertices, blocks_for(m.nVerts, 128), 128, 0, st, m, rkVal);
}

void launch_motion_geometry(const MotionArgs &m, bool transforms, cudaStream_t st) {
  const long long n = (long long)(m.nS + m.nFp) * m.E;
  if (m.nDims == 2)
    launch_k(k_motion_geometry<2>, blocks_for(n, 128), 128, 0, st, m, (int)transforms);
  else
    launch_k(k_motion_geometry<3>, blocks_for(n, 128), 128, 0, st, m, (int)transforms);
}

void launch_face_refresh(const FaceTableT<double> &ft, int nDims, const double *norm, const double *dA,
                         cudaStream_t st) {
  if (ft.n <= 0) return;
  launch_k(k_face_refresh, blocks_for(ft.n, 256), 256, 0, st, ft.n, nDims, ft.slotL, ft.slotR, norm, dA,
           const_cast<double *>(ft.nrm), const_cast<double *>(ft.dAL), const_cast<double *>(ft.dAR));
}

void launch_faces_motion(int nDims, const FaceTableT<double> &ft, const double *Uf, double *Fn, double *waveSp,
                         const double *gVf, const Phys &ph, cudaStream_t st) {
  if (ft.n <= 0) return;
  if (nDims == 2)
    launch_k(k_faces_motion<2>, blocks_for(ft.n, 256), 256, 0, st, ft, Uf, Fn, waveSp, gVf, ph);
  else
    launch_k(k_faces_motion<3>, blocks_for(ft.n, 256), 256, 0, st, ft, Uf, Fn, waveSp, gVf, ph);
}

void launch_wavesp_motion(int nDims, int nFp, int E, const double *Uf, const double *norm, const double *gVf,
                          double gamma, double *waveSp, cudaStream_t st) {
  const long long n = (long long)nFp * E;
  if (n <= 0) return;
  if (nDims == 2)
    launch_k(k_wavesp_motion<2>, blocks_for(n, 256), 256, 0, st, nFp, E, Uf, norm, gVf, gamma, waveSp);
  else
    launch_k(k_wavesp_motion<3>, blocks_for(n, 256), 256, 0, st, nFp, E, Uf, norm, gVf, gamma, waveSp);
}

void launch_motion_residual(const MotionArgs &m, const double *U, const double *Fn, double gamma, double *F,
                            double *disFn, double *divF, cudaStream_t st) {
  const long long nSE = (long long)m.nS * m.E, nFE = (long long)m.nFp * m.E;
  if (nSE <= 0) return;
  if (m.nDims == 2) {
    launch_k(k_motion_flux<2>, blocks_for(nSE, 256), 256, 0, st, m.nS, m.E, U, gamma, F);
    launch_k(k_motion_divergence<2>, blocks_for(nSE, 128), 128, 0, st, m, U, (const double *)F, divF);
    launch_k(k_motion_normal_flux<2>, blocks_for(nFE, 128), 128, 0, st, m, (const double *)F, Fn, disFn);
    launch_k(k_motion_correct<2>, blocks_for(nSE, 128), 128, 0, st, m, (const double *)disFn, divF);
  } else {
    launch_k(k_motion_flux<3>, blocks_for(nSE, 256), 256, 0, st, m.nS, m.E, U, gamma, F);
    launch_k(k_motion_divergence<3>, blocks_for(nSE, 128), 128, 0, st, m, U, (const double *)F, divF);
    launch_k(k_motion_normal_flux<3>, blocks_for(nFE, 128), 128, 0, st, m, (const double *)F, Fn, disFn);
    launch_k(k_motion_correct<3>, blocks_for(nSE, 128), 128, 0, st, m, (const double *)disFn, divF);
  }
}

void launch_motion_step_a(long long nSE, int nF, int E, const double *U0, const double *divF, const double *src,
                          const double *detJ, const double *dt, const double *eleDt, double rk, double *U,
                          cudaStream_t st) {
  const long long n = nSE * nF;
  if (n > 0)
    launch_k(k_motion_step_a, blocks_for(n, 256), 256, 0, st, nSE, nF, E, U0, divF, src, detJ, dt, eleDt, rk, U);
}

void launch_motion_step_b(long long nSE, int nF, int E, const double *base, const MotionStages &stages,
                          const double *src, const double *detJ, const double *dt, const double *eleDt, double *U,
                          cudaStream_t st) {
  const long long n = nSE * nF;
  if (n > 0)
    launch_k(k_motion_step_b, blocks_for(n, 256), 256, 0, st, nSE, nF, E, base, stages, src, detJ, dt, eleDt, U);
}

}  // namespace frk
