// Viscous (LDG) pieces of a stage, FP64 plain form and FP32 precision form
// (reference: solver.cpp:366-445 with viscous = 1):
//   k_faces_ldg_*   LDG interface solution UC and the jumps dUc = UC - U at
//                   both sides of every face point (face.cpp:188-202, 588-615);
//   k_elem_grad     corrected gradient at the solution points, transformed to
//                   physical space (solver.cpp:1060-1137), and its extrapolation
//                   to the flux points (solver.cpp:1139-1158);
//   k_faces_visc_*  inviscid + LDG viscous common flux, times dA, at both sides
//                   (face.cpp:163-186, 210-311; boundFace.cpp:316-350).
// The viscous flux at the solution points is added in the element kernel.
#include "launch.cuh"
#include "stage.hpp"

namespace frk {

namespace {

constexpr int ipow3(int b, int e) { return e == 0 ? 1 : b * ipow3(b, e - 1); }

// LDG penalty direction switch (face.cpp:596-604, 244-252).
template <int ND, typename R>
__device__ __forceinline__ R ldg_pen(const R *n, R penFact) {
  if (ND == 2) return (n[0] + n[1] < 0) ? -penFact : penFact;
  return (n[0] + n[1] + sqrt(R(2.)) * n[ND - 1] < 0) ? -penFact : penFact;
}

// One thread per (interior face point, field): the jumps of one field need
// only that field's two traces, so consecutive threads read and write
// consecutive words.
template <int ND, typename R>
__global__ void k_faces_ldg_interior(int n, const int *__restrict__ slotL, const int *__restrict__ slotR,
                                     const R *__restrict__ nrm, const R *__restrict__ Uf,
                                     R *__restrict__ dUc, R penFact) {
  pdl_wait();
  pdl_trigger();
  constexpr int NF = ND + 2;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)n * NF) return;
  const int i = (int)(t / NF), k = (int)(t - (long long)i * NF);
  const int sL = slotL[i], sR = slotR[i];
  R nv[ND];
#pragma unroll
  for (int d = 0; d < ND; d++) nv[d] = nrm[(long long)i * ND + d];
  const R pen = ldg_pen<ND, R>(nv, penFact);
  const R ul = Uf[(long long)sL * NF + k], ur = Uf[(long long)sR * NF + k];
  const R uc = R(0.5) * (ul + ur) - pen * (ul - ur);
  dUc[(long long)sL * NF + k] = uc - ul;
  dUc[(long long)sR * NF + k] = uc - ur;
}

template <int ND, typename R>
__global__ void k_faces_ldg_boundary(int n0, int n, const int *__restrict__ slotL, const int *__restrict__ slotR,
                                     const R *__restrict__ nrm, const R *__restrict__ Uf,
                                     R *__restrict__ dUc, Phys ph) {
  pdl_wait();
  pdl_trigger();
  constexpr int NF = ND + 2;
  int i = n0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int sL = slotL[i];
  const int bc = -slotR[i] - 2;
  R UL[NF], UR[NF], nv[ND];
#pragma unroll
  for (int k = 0; k < NF; k++) UL[k] = Uf[(long long)sL * NF + k];
#pragma unroll
  for (int d = 0; d < ND; d++) nv[d] = nrm[(long long)i * ND + d];
  boundary_state<ND, R>(bc, UL, nv, ph, UR);
#pragma unroll
  for (int k = 0; k < NF; k++) {
    const R uc = R(0.5) * (UL[k] + UR[k]);
    dUc[(long long)sL * NF + k] = uc - UL[k];
  }
}

// Common viscous flux added to the inviscid one (face.cpp:216-287), then *dA.
template <int ND, typename R>
__device__ __forceinline__ void ldg_interior_flux(const R *UL, const R *UR,
                                                  const R gL[ND][ND + 2], const R gR[ND][ND + 2],
                                                  const R *n, const Phys &ph, R *Fn) {
  constexpr int NF = ND + 2;
  R FL[ND][NF], FR[ND][NF];
  viscous_flux<ND, R>(UL, gL, ph, FL);
  viscous_flux<ND, R>(UR, gR, ph, FR);
  const R pen = ldg_pen<ND, R>(n, R(ph.penFact));
  const R nx = n[0], ny = n[1], nz = ND == 3 ? n[ND - 1] : R(0.0);
  R Fc[ND][NF];
#pragma unroll
  for (int k = 0; k < NF; k++) {
    const R dF0 = FL[0][k] - FR[0][k];
    const R dF1 = FL[1][k] - FR[1][k];
    const R dU = UL[k] - UR[k];
    if (ND == 2) {
      Fc[0][k] = R(0.5) * (FL[0][k] + FR[0][k]) + pen * nx * (nx * (dF0) + ny * (dF1)) + R(ph.tau) * nx * (dU);
      Fc[1][k] = R(0.5) * (FL[1][k] + FR[1][k]) + pen * ny * (nx * (dF0) + ny * (dF1)) + R(ph.tau) * ny * (dU);
    } else {
      // the reference pairs the left y-flux with the right z-flux here
      // (face.cpp:277); reproduced unless the quirk switch is off
      const R dF2 = ph.viscFluxQuirk ? FL[1][k] - FR[ND - 1][k] : FL[ND - 1][k] - FR[ND - 1][k];
      const R s = nx * (dF0) + ny * (dF1) + nz * (dF2);
      Fc[0][k] = R(0.5) * (FL[0][k] + FR[0][k]) + pen * nx * s + R(ph.tau) * nx * (dU);
      Fc[1][k] = R(0.5) * (FL[1][k] + FR[1][k]) + pen * ny * s + R(ph.tau) * ny * (dU);
      Fc[ND - 1][k] = R(0.5) * (FL[ND - 1][k] + FR[ND - 1][k]) + pen * nz * s + R(ph.tau) * nz * (dU);
    }
  }
#pragma unroll
  for (int d = 0; d < ND; d++)
#pragma unroll
    for (int k = 0; k < NF; k++) Fn[k] += Fc[d][k] * n[d];
}

// Registers capped for four 128-thread CTAs per SM: the FP64 3-D kernel
// needs 148 uncapped (three CTAs) and spills 48 bytes at 128 (NS TGV 40^3
// P4 face pass 1.707 -> 1.659 ms; a cap of 96, 196 bytes spilled, is
// slower); the FP32 and 2-D kernels are below the cap.
template <int ND, typename R>
__global__ void __launch_bounds__(128, 4) k_faces_visc_interior(int n, const int *__restrict__ slotL, const int *__restrict__ slotR,
                                      const R *__restrict__ nrm, const R *__restrict__ dAL,
                                      const R *__restrict__ dAR, const R *__restrict__ Uf,
                                      const R *__restrict__ dUf, long long dStride, R *__restrict__ Fn,
                                      double *__restrict__ waveSp, Phys ph) {
  pdl_wait();
  pdl_trigger();
  constexpr int NF = ND + 2;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int sL = slotL[i], sR = slotR[i];
  R UL[NF], UR[NF], nv[ND], F[NF], gL[ND][NF], gR[ND][NF];
#pragma unroll
  for (int k = 0; k < NF; k++) {
    UL[k] = Uf[(long long)sL * NF + k];
    UR[k] = Uf[(long long)sR * NF + k];
  }
#pragma unroll
  for (int d = 0; d < ND; d++) {
    nv[d] = nrm[(long long)i * ND + d];
#pragma unroll
    for (int k = 0; k < NF; k++) {
      gL[d][k] = dUf[d * dStride + (long long)sL * NF + k];
      gR[d][k] = dUf[d * dStride + (long long)sR * NF + k];
    }
  }
  if (ND == 2 && ph.riemannType == 1) {
    roe2d<R>(UL, UR, nv, R(ph.gamma), F);
  } else {
    const R ws = rusanov<ND, R>(UL, UR, nv, R(ph.gamma), F);
    if (waveSp) waveSp[sL] = ws;  // null when no CFL time step reads it
  }
  ldg_interior_flux<ND, R>(UL, UR, gL, gR, nv, ph, F);
  const R aL = dAL[i], aR = dAR[i];
  // the left record, then the right one (stores interleaved field by field
  // between the two records measured 20-30 % slower in the inviscid kernel)
#pragma unroll
  for (int k = 0; k < NF; k++) Fn[(long long)sL * NF + k] = F[k] * aL;
#pragma unroll
  for (int k = 0; k < NF; k++) Fn[(long long)sR * NF + k] = -F[k] * aR;
}

template <int ND, typename R>
__global__ void k_faces_visc_boundary(int n0, int n, const int *__restrict__ slotL,
                                      const int *__restrict__ slotR, const R *__restrict__ nrm,
                                      const R *__restrict__ dAL, const R *__restrict__ Uf,
                                      const R *__restrict__ dUf, long long dStride, R *__restrict__ Fn,
                                      double *__restrict__ waveSp, Phys ph) {
  pdl_wait();
  pdl_trigger();
  constexpr int NF = ND + 2;
  int i = n0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int sL = slotL[i];
  const int bc = -slotR[i] - 2;
  R UL[NF], UR[NF], nv[ND], F[NF], g[ND][NF];
#pragma unroll
  for (int k = 0; k < NF; k++) UL[k] = Uf[(long long)sL * NF + k];
#pragma unroll
  for (int d = 0; d < ND; d++) {
    nv[d] = nrm[(long long)i * ND + d];
#pragma unroll
    for (int k = 0; k < NF; k++) g[d][k] = dUf[d * dStride + (long long)sL * NF + k];
  }
  boundary_state<ND, R>(bc, UL, nv, ph, UR);
  const R ws = rusanov<ND, R>(UL, UR, nv, R(ph.gamma), F);
  if (waveSp) waveSp[sL] = ws;
  R Fv[ND][NF];
  if (bc == BC_ADI_NOSLIP) {
    // adiabatic wall: right gradient with the temperature gradient removed
    // (boundFace.cpp:316-350), right-state viscous flux
    const R gam = R(ph.gamma);
    R rhovSq = R(0.);
#pragma unroll
    for (int d = 0; d < ND; d++) rhovSq += UL[d + 1] * UL[d + 1];
    const R pL = (gam - R(1.)) * (UL[ND + 1] - R(0.5) * rhovSq / UL[0]);
    const R pR = pL;
    const R e = pR / ((gam - R(1.)) * UR[0]);
    R gradVel[ND][ND];
#pragma unroll
    for (int d1 = 0; d1 < ND; d1++)
#pragma unroll
      for (int d2 = 0; d2 < ND; d2++) gradVel[d1][d2] = (g[d1][d2 + 1] - g[d1][0] * UR[d2 + 1] / UR[0]) / UR[0];
    R vSq = R(0.);
#pragma unroll
    for (int d = 0; d < ND; d++) vSq += UR[d + 1] * UR[d + 1] / (UR[0] * UR[0]);
#pragma unroll
    for (int d1 = 0; d1 < ND; d1++) {
      R v = (e + R(0.5) * vSq) * g[d1][0];
#pragma unroll
      for (int d2 = 0; d2 < ND; d2++) v += UR[d2 + 1] * gradVel[d2][d1];
      g[d1][ND + 1] = v;
    }
    viscous_flux<ND, R>(UR, g, ph, Fv);
  } else {
    viscous_flux<ND, R>(UL, g, ph, Fv);
  }
#pragma unroll
  for (int d = 0; d < ND; d++)
#pragma unroll
    for (int k = 0; k < NF; k++) Fv[d][k] = Fv[d][k] + R(ph.tau) * nv[d] * (UL[k] - UR[k]);
#pragma unroll
  for (int d = 0; d < ND; d++)
#pragma unroll
    for (int k = 0; k < NF; k++) F[k] += Fv[d][k] * nv[d];
  const R aL = dAL[i];
#pragma unroll
  for (int k = 0; k < NF; k++) Fn[(long long)sL * NF + k] = F[k] * aL;
}

// Corrected, physical solution gradient at the solution points and at the
// flux points, tensor-product form, one thread per (solution point, element).
template <int ND, int P, typename R>
struct Tg {
  static constexpr int N = P + 1;
  static constexpr int NF = ND + 2;
  static constexpr int NS = ipow3(N, ND);
  static constexpr int NFP = 2 * ND * ipow3(N, ND - 1);
  static constexpr int EB = NS >= 128 ? 1 : (NS * 2 > 128 ? 1 : (NS * 4 > 128 ? 2 : (NS * 8 > 128 ? 4 : (NS * 16 > 128 ? 8 : (NS * 32 > 128 ? 16 : 32)))));
  static constexpr int NT = NS * EB;
  static constexpr int ROW = EB * NF;
  static constexpr bool PAIR = NFP * EB > NT;  // extrapolation per line (both ends)
  static constexpr size_t SMEM = sizeof(R) * ((size_t)ROW * (NS * (1 + ND) + NFP) + N * N + 2 * N);
};

template <int ND, int P, typename R>
__global__ void __launch_bounds__(Tg<ND, P, R>::NT) k_elem_grad(GradArgsT<R> g, TpTablesT<R> t) {
  pdl_wait();
  pdl_trigger();
  using T = Tg<ND, P, R>;
  constexpr int N = T::N, NF = T::NF, NS = T::NS, NFP = T::NFP, EB = T::EB, NT = T::NT, ROW = T::ROW;
  extern __shared__ __align__(16) unsigned char smem_bytes[];
  R *smem = reinterpret_cast<R *>(smem_bytes);
  R *sU = smem;                 // [NS][ROW]
  R *sG = sU + NS * ROW;        // [ND][NS][ROW] physical gradient
  R *sC = sG + ND * NS * ROW;   // [NFP][ROW] dUc
  R *sD = sC + NFP * ROW;
  R *sE = sD + N * N;
  const int E = g.E;
  const int e0 = blockIdx.x * EB;
  const int nValid = min(EB, E - e0);
  const int tid = threadIdx.x;
  const int s = tid / EB, el = tid - (tid / EB) * EB;
  const int e = e0 + el;
  const bool valid = el < nValid;
  for (int i = tid; i < N * N; i += NT) sD[i] = t.D[i];
  for (int i = tid; i < 2 * N; i += NT) sE[i] = t.E1[i];
  for (int idx = tid; idx < NS * ROW; idx += NT) {
    const int ss = idx / ROW, r = idx - ss * ROW;
    sU[idx] = (r < nValid * NF) ? g.U[((long long)ss * E + e0) * NF + r] : R(0.0);
  }
  for (int idx = tid; idx < NFP * ROW; idx += NT) {
    const int f = idx / ROW, r = idx - f * ROW;
    sC[idx] = (r < nValid * NF) ? g.dUc[((long long)f * E + e0) * NF + r] : R(0.0);
  }
  R J[ND][ND];
#pragma unroll
  for (int d1 = 0; d1 < ND; d1++)
#pragma unroll
    for (int d2 = 0; d2 < ND; d2++) J[d1][d2] = valid ? g.JGinv[(((long long)d1 * NS + s) * E + e) * ND + d2] : R(0.0);
  const R invDet = valid ? R(1.) / g.detJ[(long long)s * E + e] : R(0.0);
  __syncthreads();

  int idx3[3];
  idx3[0] = s % N;
  idx3[1] = ND > 1 ? (s / N) % N : 0;
  idx3[2] = ND > 2 ? s / (N * N) : 0;
  R gr[ND][NF];
#pragma unroll
  for (int d = 0; d < ND; d++) {
    const int stride = d == 0 ? 1 : (d == 1 ? N : N * N);
    const int base = s - idx3[d] * stride;
    const R *Dr = &sD[idx3[d] * N];
    R acc[NF];
#pragma unroll
    for (int k = 0; k < NF; k++) acc[k] = R(0.0);
#pragma unroll
    for (int m = 0; m < N; m++) {
      const R dv = Dr[m];
      const R *x = &sU[(base + m * stride) * ROW + el * NF];
#pragma unroll
      for (int k = 0; k < NF; k++) acc[k] += dv * x[k];
    }
    // + opp_correctU[d] . dUc: the faces normal to d, ascending
    R cq[NF];
#pragma unroll
    for (int k = 0; k < NF; k++) cq[k] = R(0.0);
#pragma unroll
    for (int fc = 0; fc < 2 * ND; fc++) {
      const int fp = __ldg(&t.corrFpt[s * 2 * ND + fc]);
      if (__ldg(&t.fptDn[fp]) != d) continue;
      const R cv = __ldg(&t.corrVal[s * 2 * ND + fc]) * (__ldg(&t.fptSide[fp]) ? R(1.0) : -R(1.0));
      const R *x = &sC[fp * ROW + el * NF];
#pragma unroll
      for (int k = 0; k < NF; k++) cq[k] += cv * x[k];
    }
#pragma unroll
    for (int k = 0; k < NF; k++) gr[d][k] = cq[k] + acc[k];
  }
  // physical gradient (solver.cpp:1101-1134)
#pragma unroll
  for (int d2 = 0; d2 < ND; d2++)
#pragma unroll
    for (int k = 0; k < NF; k++) {
      R v = gr[0][k] * J[0][d2] + gr[1][k] * J[1][d2];
      if (ND == 3) v = gr[0][k] * J[0][d2] + gr[1][k] * J[1][d2] + gr[ND - 1][k] * J[ND - 1][d2];
      v = invDet * v;
      sG[(d2 * NS + s) * ROW + el * NF + k] = v;
      if (valid) g.dUs[(long long)d2 * g.sStride + ((long long)s * E + e) * NF + k] = v;
    }
  __syncthreads();
  // per flux point, or (PAIR) per line: both ends from one pass over it
  constexpr int NE = T::PAIR ? 2 : 1;
  for (int it = tid; it < (NFP / NE) * EB; it += NT) {
    const int l = it / EB, fe = it - (it / EB) * EB;
    if (fe >= nValid) continue;
    const int pr = T::PAIR ? __ldg(&t.linePair[l]) : l;
    const int f0 = pr & 0xffff;
    const int base = __ldg(&t.fptBase[f0]), dn = __ldg(&t.fptDn[f0]);
    const int side0 = T::PAIR ? 0 : __ldg(&t.fptSide[f0]);
    const int stride = dn == 0 ? 1 : (dn == 1 ? N : N * N);
#pragma unroll
    for (int d = 0; d < ND; d++) {
      R acc[NE][NF];
#pragma unroll
      for (int j = 0; j < NE; j++)
#pragma unroll
        for (int k = 0; k < NF; k++) acc[j][k] = R(0.0);
#pragma unroll
      for (int m = 0; m < N; m++) {
        const R *x = &sG[(d * NS + base + m * stride) * ROW + fe * NF];
#pragma unroll
        for (int j = 0; j < NE; j++) {
          const R ev = sE[(j ? 1 : side0) * N + m];
#pragma unroll
          for (int k = 0; k < NF; k++) acc[j][k] += ev * x[k];
        }
      }
#pragma unroll
      for (int j = 0; j < NE; j++) {
        const int f = j ? pr >> 16 : f0;
#pragma unroll
        for (int k = 0; k < NF; k++) g.dUf[(long long)d * g.fStride + ((long long)f * E + e0 + fe) * NF + k] = acc[j][k];
      }
    }
  }
}

template <int ND, int P, typename R>
void launch_grad(const GradArgsT<R> &g, const TpTablesT<R> &t, cudaStream_t st) {
  using T = Tg<ND, P, R>;
  static std::atomic<unsigned long long> attrDev{0};
  smem_attr(k_elem_grad<ND, P, R>, (int)T::SMEM, attrDev);
  launch_k(k_elem_grad<ND, P, R>, (g.E + T::EB - 1) / T::EB, T::NT, T::SMEM, st, g, t);
}

}  // namespace

template <typename R>
void launch_faces_ldg(int nDims, const FaceTableT<R> &ft, const R *Ufpts, R *dUc, const Phys &ph, cudaStream_t st) {
  const int b = 256, nI = ft.nInterior, nB = ft.n - ft.nInterior;
  if (nI > 0) {
    const long long nt = (long long)nI * (nDims + 2);
    const unsigned g = (unsigned)((nt + b - 1) / b);
    if (nDims == 2)
      launch_k(k_faces_ldg_interior<2, R>, g, b, 0, st, nI, ft.slotL, ft.slotR, ft.nrm, Ufpts, dUc, ph.penFact);
    else
      launch_k(k_faces_ldg_interior<3, R>, g, b, 0, st, nI, ft.slotL, ft.slotR, ft.nrm, Ufpts, dUc, ph.penFact);
  }
  if (nB > 0) {
    if (nDims == 2)
      launch_k(k_faces_ldg_boundary<2, R>, (nB + b - 1) / b, b, 0, st, nI, ft.n, ft.slotL, ft.slotR, ft.nrm, Ufpts, dUc, ph);
    else
      launch_k(k_faces_ldg_boundary<3, R>, (nB + b - 1) / b, b, 0, st, nI, ft.n, ft.slotL, ft.slotR, ft.nrm, Ufpts, dUc, ph);
  }
}

template <typename R>
void launch_faces_visc(int nDims, const FaceTableT<R> &ft, const R *Ufpts, const R *dUf, long long fStride, R *Fn,
                       double *waveSp, const Phys &ph, cudaStream_t st) {
  const int b = 128, nI = ft.nInterior, nB = ft.n - ft.nInterior;
  if (nI > 0) {
    if (nDims == 2)
      launch_k(k_faces_visc_interior<2, R>, (nI + b - 1) / b, b, 0, st, nI, ft.slotL, ft.slotR, ft.nrm, ft.dAL, ft.dAR, Ufpts,
                                                               dUf, fStride, Fn, waveSp, ph);
    else
      launch_k(k_faces_visc_interior<3, R>, (nI + b - 1) / b, b, 0, st, nI, ft.slotL, ft.slotR, ft.nrm, ft.dAL, ft.dAR, Ufpts,
                                                               dUf, fStride, Fn, waveSp, ph);
  }
  if (nB > 0) {
    if (nDims == 2)
      launch_k(k_faces_visc_boundary<2, R>, (nB + b - 1) / b, b, 0, st, nI, ft.n, ft.slotL, ft.slotR, ft.nrm, ft.dAL, Ufpts,
                                                               dUf, fStride, Fn, waveSp, ph);
    else
      launch_k(k_faces_visc_boundary<3, R>, (nB + b - 1) / b, b, 0, st, nI, ft.n, ft.slotL, ft.slotR, ft.nrm, ft.dAL, Ufpts,
                                                               dUf, fStride, Fn, waveSp, ph);
  }
}

template <typename R>
void launch_elem_grad(int nDims, int order, const GradArgsT<R> &g, const TpTablesT<R> &t, cudaStream_t st) {
  if (g.E <= 0) return;
#define FR_G_CASE(ND, P) \
  if (nDims == ND && order == P) return launch_grad<ND, P, R>(g, t, st);
  FR_G_CASE(2, 0) FR_G_CASE(2, 1) FR_G_CASE(2, 2) FR_G_CASE(2, 3) FR_G_CASE(2, 4) FR_G_CASE(2, 5)
  FR_G_CASE(3, 0) FR_G_CASE(3, 1) FR_G_CASE(3, 2) FR_G_CASE(3, 3) FR_G_CASE(3, 4) FR_G_CASE(3, 5)
#undef FR_G_CASE
}

#define FR_VISC_INST(R)                                                                                    \
  template void launch_faces_ldg<R>(int, const FaceTableT<R> &, const R *, R *, const Phys &, cudaStream_t);      \
  template void launch_faces_visc<R>(int, const FaceTableT<R> &, const R *, const R *, long long, R *, double *, \
                                     const Phys &, cudaStream_t);                                                \
  template void launch_elem_grad<R>(int, int, const GradArgsT<R> &, const TpTablesT<R> &, cudaStream_t);
FR_VISC_INST(double)
FR_VISC_INST(float)
#undef FR_VISC_INST

}  // namespace frk
