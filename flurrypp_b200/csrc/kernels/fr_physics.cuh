// Point-wise physics on the device: Euler flux, common (Riemann) fluxes,
// boundary ghost states, LDG viscous flux.  Each function restates the
// reference's arithmetic in the same operation order, so the FP64 form
// differs from the reference CPU build only by FMA contraction and operator
// application order (<= a few ulp per point).
#pragma once
#include <cuda_runtime.h>

namespace frk {

// Boundary-condition codes (reference: include/global.hpp:116-132).
enum : int {
  BC_PERIODIC = 0,
  BC_CHAR = 1,
  BC_SUP_IN = 2,
  BC_SUP_OUT = 3,
  BC_SUB_IN = 4,
  BC_SUB_OUT = 5,
  BC_SLIP_WALL = 8,
  BC_ISO_NOSLIP = 9,
  BC_ADI_NOSLIP = 10,
  BC_SYMMETRY = 12,
  BC_ISO_NOSLIP_MOVING = 13
};

// Per-case physical constants the kernels need.
struct Phys {
  double gamma;
  double rhoBound, uBound, vBound, wBound, pBound;
  double TWall, RGas, uWall, vWall, wWall;
  // viscous
  double mu_inf, prandtl, rt_inf, c_sth, penFact, tau;
  int fixVis;
  int viscFluxQuirk;  // 1: the reference's 3-D stress/flux formulas (flux.cpp:184-201)
  int riemannType;    // 0 Rusanov, 1 Roe (2-D interior faces only)
};

// Euler flux F[d][k] (reference: src/flux.cpp:37-76).
template <int ND, typename R>
__device__ __forceinline__ void inviscid_flux(const R *U, R F[ND][ND + 2], R gam) {
  if (ND == 2) {
    R rho = U[0];
    R ri = R(1.0) / rho;
    R u = U[1] * ri;
    R v = U[2] * ri;
    R E = U[3];
    R p = (gam - R(1.0)) * (E - R(0.5) * rho * (u * u + v * v));
    F[0][0] = rho * u;          F[1][0] = rho * v;
    F[0][1] = rho * u * u + p;  F[1][1] = rho * u * v;
    F[0][2] = rho * v * u;      F[1][2] = rho * v * v + p;
    F[0][3] = (E + p) * u;      F[1][3] = (E + p) * v;
  } else {
    R rho = U[0];
    R ri = R(1.0) / rho;
    R u = U[1] * ri;
    R v = U[2] * ri;
    R w = U[3] * ri;
    R E = U[4];
    R p = (gam - R(1.0)) * (E - R(0.5) * rho * (u * u + v * v + w * w));
    F[0][0] = rho * u;          F[1][0] = rho * v;          F[ND - 1][0] = rho * w;
    F[0][1] = rho * u * u + p;  F[1][1] = rho * u * v;      F[ND - 1][1] = rho * u * w;
    F[0][2] = rho * v * u;      F[1][2] = rho * v * v + p;  F[ND - 1][2] = rho * v * w;
    F[0][3] = rho * w * u;      F[1][3] = rho * w * v;      F[ND - 1][3] = rho * w * w + p;
    F[0][4] = (E + p) * u;      F[1][4] = (E + p) * v;      F[ND - 1][4] = (E + p) * w;
  }
}

// Primitive state used by the common fluxes: velocity, pressure, energy, with
// the operations of inviscidFlux (reference: src/flux.cpp:37-76).
template <int ND, typename R>
struct Prim {
  R rho, vel[ND], E, p;
  R rinv;
  __device__ __forceinline__ Prim(const R *U, R gam) {
    rho = U[0];
    rinv = R(1.0) / rho;  // one reciprocal per state instead of a division per term
#pragma unroll
    for (int d = 0; d < ND; d++) vel[d] = U[d + 1] * rinv;
    E = U[ND + 1];
    R q = vel[0] * vel[0] + vel[1] * vel[1];
    if (ND == 3) q = vel[0] * vel[0] + vel[1] * vel[1] + vel[ND - 1] * vel[ND - 1];
    p = (gam - R(1.0)) * (E - R(0.5) * rho * q);
  }
  // flux along dimension d, F[d][k] of inviscidFlux
  __device__ __forceinline__ void flux(int d, R *F) const {
    F[0] = rho * vel[d];
#pragma unroll
    for (int j = 0; j < ND; j++) F[1 + j] = j == d ? rho * vel[j] * vel[d] + p : rho * vel[j] * vel[d];
    F[ND + 1] = (E + p) * vel[d];
  }
};

// Rusanov common flux on the left normal; returns the wave speed stored for
// the dt estimate (reference: src/face.cpp:314-374).
template <int ND, typename R>
__device__ __forceinline__ R rusanov(const R *UL, const R *UR, const R *n, R gam, R *Fn, R vgn = R(0)) {
  constexpr int NF = ND + 2;
  const Prim<ND, R> L(UL, gam), Rt(UR, gam);
  R vnL = R(0), vnR = R(0);
  R tL[NF], tR[NF];
#pragma unroll
  for (int i = 0; i < NF; i++) tL[i] = tR[i] = R(0);
#pragma unroll
  for (int d = 0; d < ND; d++) {
    vnL += n[d] * L.vel[d];
    vnR += n[d] * Rt.vel[d];
    R f[NF];
    L.flux(d, f);
#pragma unroll
    for (int i = 0; i < NF; i++) tL[i] += n[d] * f[i];
    Rt.flux(d, f);
#pragma unroll
    for (int i = 0; i < NF; i++) tR[i] += n[d] * f[i];
  }
  R csqL = fmax(gam * L.p * L.rinv, R(0.0));
  R csqR = fmax(gam * Rt.p * Rt.rinv, R(0.0));
  R eigL = fabs(vnL) + sqrt(csqL);
  R eigR = fabs(vnR) + sqrt(csqR);
  R eig = fmax(eigL, eigR);
#pragma unroll
  for (int i = 0; i < NF; i++) Fn[i] = R(0.5) * (tL[i] + tR[i] - eig * (UR[i] - UL[i]));
  // the wave speed kept for the time step is relative to the grid velocity
  // on a moving mesh (face.cpp:366-371; vgn is zero on a static one)
  return fmax(fabs(vnL - vgn) + sqrt(csqL), fabs(vnR - vgn) + sqrt(csqR));
}

// Roe flux with entropy fix, 2-D (reference: src/face.cpp:376-495).
template <typename R>
__device__ __forceinline__ void roe2d(const R *UL, const R *UR, const R *n, R gamma, R *Fn) {
  const int nDims = 2;
  R vL[2], vR[2], um[2], du[4];
  for (int i = 0; i < nDims; i++) {
    vL[i] = UL[i + 1] / UL[0];
    vR[i] = UR[i + 1] / UR[0];
  }
  R pL = (gamma - R(1.0)) * (UL[3] - (R(0.5) * UL[0] * (vL[0] * vL[0] + vL[1] * vL[1])));
  R pR = (gamma - R(1.0)) * (UR[3] - (R(0.5) * UR[0] * (vR[0] * vR[0] + vR[1] * vR[1])));
  R hL = (UL[nDims + 1] + pL) / UL[0];
  R hR = (UR[nDims + 1] + pR) / UR[0];
  R sq_rho = sqrt(UR[0] / UL[0]);
  R rrho = R(1.) / (sq_rho + R(1.));
  R usq = R(0.), unm = R(0.);
  for (int i = 0; i < nDims; i++) {
    um[i] = rrho * (vL[i] + sq_rho * vR[i]);
    usq += R(0.5) * um[i] * um[i];
    unm += um[i] * n[i];
  }
  R hm = rrho * (hL + sq_rho * hR);
  R am_sq = (gamma - R(1.)) * (hm - usq);
  R am = sqrt(am_sq);
  R rhoUnL = R(0.), rhoUnR = R(0.);
  for (int i = 0; i < nDims; i++) {
    rhoUnL += UL[i + 1] * n[i];
    rhoUnR += UR[i + 1] * n[i];
  }
  Fn[0] = rhoUnL + rhoUnR;
  Fn[1] = rhoUnL * vL[0] + rhoUnR * vR[0] + (pL + pR) * n[0];
  Fn[2] = rhoUnL * vL[1] + rhoUnR * vR[1] + (pL + pR) * n[1];
  Fn[3] = rhoUnL * hL + rhoUnR * hR;
  for (int i = 0; i < 4; i++) du[i] = UR[i] - UL[i];
  R lambda0 = fabs(unm);
  R lambdaP = fabs(unm + am);
  R lambdaM = fabs(unm - am);
  R eps = R(0.5) * (fabs(rhoUnL / UL[0] - rhoUnR / UR[0]) +
                    fabs(sqrt(gamma * pL / UL[0]) - sqrt(gamma * pR / UR[0])));
  if (lambda0 < R(2.) * eps) lambda0 = R(0.25) * lambda0 * lambda0 / eps + eps;
  if (lambdaP < R(2.) * eps) lambdaP = R(0.25) * lambdaP * lambdaP / eps + eps;
  if (lambdaM < R(2.) * eps) lambdaM = R(0.25) * lambdaM * lambdaM / eps + eps;
  R a2 = R(0.5) * (lambdaP + lambdaM) - lambda0;
  R a3 = R(0.5) * (lambdaP - lambdaM) / am;
  R a1 = a2 * (gamma - R(1.)) / am_sq;
  R a4 = a3 * (gamma - R(1.));
  R a5 = usq * du[0] - um[0] * du[1] - um[1] * du[2] + du[3];
  R a6 = unm * du[0] - n[0] * du[1] - n[1] * du[2];
  R aL1 = a1 * a5 - a3 * a6;
  R bL1 = a4 * a5 - a2 * a6;
  Fn[0] -= lambda0 * du[0] + aL1;
  Fn[1] -= lambda0 * du[1] + aL1 * um[0] + bL1 * n[0];
  Fn[2] -= lambda0 * du[2] + aL1 * um[1] + bL1 * n[1];
  Fn[3] -= lambda0 * du[3] + aL1 * hm + bL1 * unm;
  for (int i = 0; i < 4; i++) Fn[i] *= R(0.5);
}

// Ghost (right) state of a boundary face (reference: src/boundFace.cpp:65-314).
// vG: the grid velocity at the point on a moving mesh (slip walls reflect the
// velocity relative to it, no-slip walls move with it); null on a static one.
template <int ND, typename R>
__device__ __forceinline__ void boundary_state(int bc, const R *UL, const R *n, const Phys &ph,
                                               R *UR, const R *vG = nullptr) {
  const R gamma = R(ph.gamma);
  const R gmo = gamma - R(1.);
  R rhoR = R(0), pR = R(0), ER = R(0);
  R vL[3] = {R(0), R(0), R(0)}, vR[3] = {R(0), R(0), R(0)};
  const R vBound[3] = {R(ph.uBound), R(ph.vBound), R(ph.wBound)};
  R rhoL = UL[0];
  R eL = UL[ND + 1];
  for (int i = 0; i < ND; i++) vL[i] = UL[i + 1] / UL[0];
  R vSq = R(0);
  for (int i = 0; i < ND; i++) vSq += (vL[i] * vL[i]);
  R pL = (gamma - R(1.0)) * (eL - R(0.5) * rhoL * vSq);
  if (bc == BC_SUB_IN) {
    rhoR = R(ph.rhoBound);
    for (int i = 0; i < ND; i++) vR[i] = vBound[i];
    pR = pL;
    vSq = R(0);
    for (int i = 0; i < ND; i++) vSq += (vR[i] * vR[i]);
    ER = (pR / (gamma - R(1.0))) + R(0.5) * rhoR * vSq;
  } else if (bc == BC_SUB_OUT) {
    rhoR = rhoL;
    for (int i = 0; i < ND; i++) vR[i] = vL[i];
    pR = R(ph.pBound);
    vSq = R(0.);
    for (int i = 0; i < ND; i++) vSq += (vR[i] * vR[i]);
    ER = (pR / (gamma - R(1.0))) + R(0.5) * rhoR * vSq;
  } else if (bc == BC_SUP_IN) {
    rhoR = R(ph.rhoBound);
    for (int i = 0; i < ND; i++) vR[i] = vBound[i];
    pR = R(ph.pBound);
    vSq = R(0.);
    for (int i = 0; i < ND; i++) vSq += (vR[i] * vR[i]);
    ER = (pR / (gamma - R(1.0))) + R(0.5) * rhoR * vSq;
  } else if (bc == BC_SUP_OUT) {
    rhoR = rhoL;
    for (int i = 0; i < ND; i++) vR[i] = vL[i];
    ER = eL;
  } else if (bc == BC_SLIP_WALL || bc == BC_SYMMETRY) {
    rhoR = rhoL;
    R vnL = R(0.);
    for (int i = 0; i < ND; i++) vnL += (vL[i] - (vG ? vG[i] : R(0))) * n[i];
    for (int i = 0; i < ND; i++) vR[i] = vL[i] - (R(2.0)) * vnL * n[i];
    ER = eL;
  } else if (bc == BC_ISO_NOSLIP_MOVING) {
    pR = pL;
    R TR = R(ph.TWall);
    rhoR = pR / (R(ph.RGas) * TR);
    vR[0] = (vG ? vG[0] : R(0)) + R(ph.uWall);
    vR[1] = (vG ? vG[1] : R(0)) + R(ph.vWall);
    if (ND == 3) vR[2] = (vG ? vG[2] : R(0)) + R(ph.wWall);
    vSq = R(0.);
    for (int i = 0; i < ND; i++) vSq += (vR[i] * vR[i]);
    ER = (pR / (gamma - R(1.0))) + R(0.5) * rhoR * vSq;
  } else if (bc == BC_ISO_NOSLIP) {
    pR = pL;
    R TR = R(ph.TWall);
    rhoR = pR / (R(ph.RGas) * TR);
    for (int i = 0; i < ND; i++) vR[i] = vG ? vG[i] : R(0);
    vSq = R(0.);
    for (int i = 0; i < ND; i++) vSq += (vR[i] * vR[i]);
    ER = (pR / (gamma - R(1.0))) + R(0.5) * rhoR * vSq;
  } else if (bc == BC_ADI_NOSLIP) {
    rhoR = rhoL;
    pR = pL;
    for (int i = 0; i < ND; i++) vR[i] = vG ? vG[i] : R(0);
    vSq = R(0.);
    for (int i = 0; i < ND; i++) vSq += (vR[i] * vR[i]);
    ER = (pR / (gamma - R(1.0))) + R(0.5) * rhoR * vSq;
  } else {  // BC_CHAR: Riemann-invariant far field
    R vnL = R(0.);
    for (int i = 0; i < ND; i++) vnL += vL[i] * n[i];
    R vnB = R(0.);
    for (int i = 0; i < ND; i++) vnB += vBound[i] * n[i];
    R cL = sqrt(gamma * pL / rhoL);
    R cB = sqrt(gamma * R(ph.pBound) / R(ph.rhoBound));
    R R_L, R_B;
    if (fabs(vnB) >= cB && vnL >= R(0))
      R_L = vnB + R(2.) / gmo * cB;
    else
      R_L = vnL + R(2.) / gmo * cL;
    if (fabs(vnB) >= cB && vnL < R(0))
      R_B = vnL - R(2.) / gmo * cL;
    else
      R_B = vnB - R(2.) / gmo * cB;
    R rhoFac = R(.25) * (gamma - R(1.)) * (R_L - R_B);
    R rhoBG = rhoFac * rhoFac / gamma;
    if (vnL < R(0))
      rhoBG *= pow(R(ph.rhoBound), gamma) / R(ph.pBound);
    else
      rhoBG *= pow(rhoL, gamma) / pL;
    rhoR = pow(rhoBG, R(1.) / gmo);
    pR = rhoFac * rhoFac * rhoR / gamma;
    R VB = R(0.5) * (R_L + R_B);
    for (int i = 0; i < ND; i++) {
      if (vnL < R(0))
        vR[i] = vBound[i] + (VB - vnB) * n[i];
      else
        vR[i] = vL[i] + (VB - vnL) * n[i];
    }
    R vMag2 = R(0);
    for (int i = 0; i < ND; i++) vMag2 += vR[i] * vR[i];
    ER = pR / gmo + R(.5) * rhoR * vMag2;
  }
  UR[0] = rhoR;
  for (int i = 0; i < ND; i++) UR[i + 1] = rhoR * vR[i];
  UR[ND + 1] = ER;
}

// Navier-Stokes viscous flux Fvis[d][k] from U and its physical gradient
// gradU[d][k] (reference: src/flux.cpp:79-210).  With ph.viscFluxQuirk the
// reference's 3-D formulas are reproduced exactly (tauxz, tauyz and the
// z-momentum entries of the x/y fluxes); without it the textbook forms.
template <int ND, typename R>
__device__ __forceinline__ void viscous_flux(const R *U, const R gradU[ND][ND + 2], const Phys &ph,
                                             R Fvis[ND][ND + 2]) {
  R rho = U[0];
  R u = U[1] / rho;
  R v = U[2] / rho;
  R e = U[ND + 1] / rho - R(0.5) * (u * u + v * v);
  R w;
  if (ND == 3) {
    w = U[3] / rho;
    e -= R(0.5) * (w * w);
  } else {
    w = R(0.);
  }
  R dRho_dx = gradU[0][0], dRhoU_dx = gradU[0][1], dRhoV_dx = gradU[0][2], dE_dx = gradU[0][ND + 1];
  R dRho_dy = gradU[1][0], dRhoU_dy = gradU[1][1], dRhoV_dy = gradU[1][2], dE_dy = gradU[1][ND + 1];
  R dRho_dz = R(0), dRhoU_dz = R(0), dRhoV_dz = R(0), dRhoW_dx = R(0), dRhoW_dy = R(0),
    dRhoW_dz = R(0), dE_dz = R(0);
  if (ND == 3) {
    dRho_dz = gradU[ND - 1][0];
    dRhoU_dz = gradU[ND - 1][1];
    dRhoV_dz = gradU[ND - 1][2];
    dRhoW_dx = gradU[0][3];
    dRhoW_dy = gradU[1][3];
    dRhoW_dz = gradU[ND - 1][3];
    dE_dz = gradU[ND - 1][4];
  }
  R mu = R(ph.mu_inf);
  if (!ph.fixVis) {
    R rt_ratio = (R(ph.gamma) - R(1.0)) * e / R(ph.rt_inf);
    mu *= pow(rt_ratio, R(1.5)) * (R(1.) + R(ph.c_sth)) / (rt_ratio + R(ph.c_sth));
  }
  R du_dx = (dRhoU_dx - dRho_dx * u) / rho;
  R du_dy = (dRhoU_dy - dRho_dy * u) / rho;
  R dv_dx = (dRhoV_dx - dRho_dx * v) / rho;
  R dv_dy = (dRhoV_dy - dRho_dy * v) / rho;
  R du_dz = R(0), dv_dz = R(0), dw_dx = R(0), dw_dy = R(0), dw_dz = R(0);
  if (ND == 3) {
    du_dz = (dRhoU_dz - dRho_dz * u) / rho;
    dv_dz = (dRhoV_dz - dRho_dz * v) / rho;
    dw_dx = (dRhoW_dx - dRho_dx * w) / rho;
    dw_dy = (dRhoW_dy - dRho_dy * w) / rho;
    dw_dz = (dRhoW_dz - dRho_dz * w) / rho;
  }
  R dK_dx, dK_dy, dK_dz;
  if (ND == 2) {
    dK_dx = R(0.5) * (u * u + v * v) * dRho_dx + rho * (u * du_dx + v * dv_dx);
    dK_dy = R(0.5) * (u * u + v * v) * dRho_dy + rho * (u * du_dy + v * dv_dy);
    dK_dz = R(0);
  } else {
    dK_dx = R(0.5) * (u * u + v * v + w * w) * dRho_dx + rho * (u * du_dx + v * dv_dx + w * dw_dx);
    dK_dy = R(0.5) * (u * u + v * v + w * w) * dRho_dy + rho * (u * du_dy + v * dv_dy + w * dw_dy);
    dK_dz = R(0.5) * (u * u + v * v + w * w) * dRho_dz + rho * (u * du_dz + v * dv_dz + w * dw_dz);
  }
  R de_dx = (dE_dx - dK_dx - dRho_dx * e) / rho;
  R de_dy = (dE_dy - dK_dy - dRho_dy * e) / rho;
  R de_dz = R(0);
  if (ND == 3) de_dz = (dE_dz - dK_dz - dRho_dz * e) / rho;
  R diag = (du_dx + dv_dy + dw_dz) / R(3.0);
  R tauxx = R(2.0) * mu * (du_dx - diag);
  R tauyy = R(2.0) * mu * (dv_dy - diag);
  R tauxy = mu * (du_dy + dv_dx);
  R tauxz = R(0), tauyz = R(0), tauzz = R(0);
  if (ND == 3) {
    if (ph.viscFluxQuirk) {
      tauxz = mu * (du_dz + dv_dx);
      tauyz = mu * (du_dz + dv_dy);
    } else {
      tauxz = mu * (du_dz + dw_dx);
      tauyz = mu * (dv_dz + dw_dy);
    }
    tauzz = R(2.0) * mu * (dw_dz - diag);
  }
  R kq = (mu / R(ph.prandtl)) * R(ph.gamma);
  Fvis[0][0] = R(0.0);
  Fvis[0][1] = -tauxx;
  Fvis[0][2] = -tauxy;
  Fvis[0][ND + 1] = -(u * tauxx + v * tauxy + w * tauxz + kq * de_dx);
  Fvis[1][0] = R(0.0);
  Fvis[1][1] = -tauxy;
  Fvis[1][2] = -tauyy;
  Fvis[1][ND + 1] = -(u * tauxy + v * tauyy + w * tauyz + kq * de_dy);
  if (ND == 3) {
    if (ph.viscFluxQuirk) {
      Fvis[0][3] = -tauzz;
      Fvis[1][3] = -tauyz;
    } else {
      Fvis[0][3] = -tauxz;
      Fvis[1][3] = -tauyz;
    }
    Fvis[ND - 1][0] = R(0.0);
    Fvis[ND - 1][1] = -tauxz;
    Fvis[ND - 1][2] = -tauyz;
    Fvis[ND - 1][3] = -tauzz;
    Fvis[ND - 1][4] = -(u * tauxz + v * tauyz + w * tauzz + kq * de_dz);
  }
}

}  // namespace frk
