// Stage kernels for sm_100a: faces, the general sparse-operator element
// kernel (FP64), time step, norms and the precision form's conversions.
//
// One RK stage is two kernels:
//   faces   : common flux Fn at every face point, gathered from U_fpts through
//             the face-point table (reference: solver.cpp:752-758);
//   element : per block of EB elements, with the element's data staged in
//             shared memory: transformed flux at the solution points
//             (solver.cpp:707-736), flux divergence (925-954), extrapolated
//             normal flux (956-1034), correction (1036-1058), the RK update
//             (470-536) and the extrapolation of the new state to the flux
//             points for the next stage's face kernel (556-572).
// Operators are applied through their nonzero entries (Csr), which for the
// tensor-product quad/hex operators removes the structural zeros of the
// reference's dense cblas_dgemm without changing any sum.
#include <algorithm>
#include <atomic>
#include <cstdio>
#include <type_traits>

#include "launch.cuh"
#include "stage.hpp"

namespace frk {

namespace {
thread_local bool g_pdl = false;
}  // namespace

void set_pdl(bool on) { g_pdl = on; }
bool pdl_enabled() { return g_pdl; }

namespace {

__global__ void k_apply_op(int nRows, const int *__restrict__ rp, const int *__restrict__ ci,
                           const double *__restrict__ v, const double *__restrict__ in,
                           double *__restrict__ out, long long N, double alpha, double beta) {
  pdl_wait();
  pdl_trigger();
  long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  int r = blockIdx.y;
  if (n >= N || r >= nRows) return;
  double s = 0.0;
  for (int j = rp[r]; j < rp[r + 1]; j++) s += v[j] * in[(long long)ci[j] * N + n];
  double o = alpha * s;
  if (beta != 0.0) o += beta * out[(long long)r * N + n];
  out[(long long)r * N + n] = o;
}

// A point's NF values in a global [slot][field] array, and a face point's
// ND normal components: in 2-D (four fields, two components, 16- or
// 32-byte and 8- or 16-byte aligned) as vector accesses, which issue a
// quarter of the memory instructions of per-value accesses; otherwise per
// value.
template <int NF, typename R>
__device__ __forceinline__ void ld_rec(const R *__restrict__ p, R (&v)[NF]) {
  if constexpr (NF == 4 && std::is_same<R, float>::value) {
    const float4 t = *reinterpret_cast<const float4 *>(p);
    v[0] = t.x, v[1] = t.y, v[2] = t.z, v[3] = t.w;
  } else if constexpr (NF == 4 && std::is_same<R, double>::value) {
    const double2 a = reinterpret_cast<const double2 *>(p)[0], b = reinterpret_cast<const double2 *>(p)[1];
    v[0] = a.x, v[1] = a.y, v[2] = b.x, v[3] = b.y;
  } else {
#pragma unroll
    for (int k = 0; k < NF; k++) v[k] = p[k];
  }
}
template <int NF, typename R>
__device__ __forceinline__ void st_rec(R *__restrict__ p, const R (&v)[NF]) {
  if constexpr (NF == 4 && std::is_same<R, float>::value) {
    *reinterpret_cast<float4 *>(p) = make_float4(v[0], v[1], v[2], v[3]);
  } else if constexpr (NF == 4 && std::is_same<R, double>::value) {
    reinterpret_cast<double2 *>(p)[0] = make_double2(v[0], v[1]);
    reinterpret_cast<double2 *>(p)[1] = make_double2(v[2], v[3]);
  } else {
#pragma unroll
    for (int k = 0; k < NF; k++) p[k] = v[k];
  }
}
template <int ND, typename R>
__device__ __forceinline__ void ld_nrm(const R *__restrict__ p, R (&v)[ND]) {
  if constexpr (ND == 2 && std::is_same<R, float>::value) {
    const float2 t = *reinterpret_cast<const float2 *>(p);
    v[0] = t.x, v[1] = t.y;
  } else if constexpr (ND == 2 && std::is_same<R, double>::value) {
    const double2 t = *reinterpret_cast<const double2 *>(p);
    v[0] = t.x, v[1] = t.y;
  } else {
#pragma unroll
    for (int d = 0; d < ND; d++) v[d] = p[d];
  }
}

// Interior face point i: Rusanov (or 2-D Roe) on the left normal, written to
// both sides (reference: face.cpp:163-208, intFace.cpp:147-154).
template <int ND, typename R>
__device__ __forceinline__ void face_interior(int i, const int *__restrict__ slotL, const int *__restrict__ slotR,
                                              const R *__restrict__ nrm, const R *__restrict__ dAL,
                                              const R *__restrict__ dAR, const R *__restrict__ Uf,
                                              R *__restrict__ Fn, double *__restrict__ waveSp, R gam, int roe) {
  constexpr int NF = ND + 2;
  const int sL = slotL[i];
  const int sR = slotR[i];
  R UL[NF], UR[NF], nv[ND], F[NF];
  ld_rec<NF, R>(&Uf[(long long)sL * NF], UL);
  ld_rec<NF, R>(&Uf[(long long)sR * NF], UR);
  ld_nrm<ND, R>(&nrm[(long long)i * ND], nv);
  if (ND == 2 && roe) {
    roe2d<R>(UL, UR, nv, gam, F);
  } else {
    const R ws = rusanov<ND, R>(UL, UR, nv, gam, F);
    if (waveSp) waveSp[sL] = ws;  // null when no CFL time step reads it
  }
  const R aL = dAL[i], aR = dAR[i];
  R FL[NF], FR[NF];
#pragma unroll
  for (int k = 0; k < NF; k++) {
    FL[k] = F[k] * aL;
    FR[k] = -F[k] * aR;
  }
  st_rec<NF, R>(&Fn[(long long)sL * NF], FL);
  st_rec<NF, R>(&Fn[(long long)sR * NF], FR);
}

// Boundary face point i: ghost state from the BC, then Rusanov (boundaries
// always use Rusanov, face.cpp:174-176; ghost states boundFace.cpp:65-314).
template <int ND, typename R>
__device__ __forceinline__ void face_boundary(int i, const int *__restrict__ slotL, const int *__restrict__ slotR,
                                              const R *__restrict__ nrm, const R *__restrict__ dAL,
                                              const R *__restrict__ Uf, R *__restrict__ Fn,
                                              double *__restrict__ waveSp, const Phys &ph) {
  constexpr int NF = ND + 2;
  const int sL = slotL[i];
  const int bc = -slotR[i] - 2;
  R UL[NF], UR[NF], nv[ND], F[NF];
  ld_rec<NF, R>(&Uf[(long long)sL * NF], UL);
  ld_nrm<ND, R>(&nrm[(long long)i * ND], nv);
  boundary_state<ND, R>(bc, UL, nv, ph, UR);
  const R ws = rusanov<ND, R>(UL, UR, nv, R(ph.gamma), F);
  if (waveSp) waveSp[sL] = ws;
  const R aL = dAL[i];
#pragma unroll
  for (int k = 0; k < NF; k++) F[k] = F[k] * aL;
  st_rec<NF, R>(&Fn[(long long)sL * NF], F);
}

// PPT face points per thread (points i and i + grid size), all gathers
// issued before any flux is formed: the gather is latency-bound, and two
// points per thread at 128 threads per CTA keep a third more loads in flight
// per SM than one point per thread at the register-limited occupancy
// (measured: 3-D FP64 faces 0.090 -> 0.083 ms, FP32 0.054 -> 0.050 ms).
// The FP64 3-D kernel's registers are capped for five CTAs per SM (118
// uncapped, 96 with 76 bytes spilled: 0.0835 -> 0.0799 ms at 32^3 P3; a cap
// of 80 for six CTAs, 124 bytes spilled, is slower, 0.0864 ms).  The FP32
// kernels are below the cap; the 2-D FP64 one (112) is left uncapped (0:
// no minimum, which leaves its register allocation as without the bound).
constexpr int kFacePpt = 2, kFaceNt = 128;
template <int ND, typename R>
constexpr int face_min_ctas() { return ND == 3 && sizeof(R) == 8 ? 5 : 0; }


template <int ND, typename R, int PPT>
__global__ void __launch_bounds__(kFaceNt, face_min_ctas<ND, R>()) k_faces_interior_ilp(int n, const int *__restrict__ slotL,
                                                           const int *__restrict__ slotR, const R *__restrict__ nrm,
                                                           const R *__restrict__ dAL, const R *__restrict__ dAR,
                                                           const R *__restrict__ Uf, R *__restrict__ Fn,
                                                           double *__restrict__ waveSp, R gam, int roe) {
  pdl_wait();
  pdl_trigger();
  constexpr int NF = ND + 2;
  const int stride = gridDim.x * blockDim.x;
  const int i0 = blockIdx.x * blockDim.x + threadIdx.x;
  int ii[PPT], sL[PPT], sR[PPT];
#pragma unroll
  for (int q = 0; q < PPT; q++) {
    ii[q] = min(i0 + q * stride, n - 1);
    sL[q] = slotL[ii[q]];
    sR[q] = slotR[ii[q]];
  }
  R UL[PPT][NF], UR[PPT][NF], nv[PPT][ND], aL[PPT], aR[PPT];
#pragma unroll
  for (int q = 0; q < PPT; q++) {
    ld_rec<NF, R>(&Uf[(long long)sL[q] * NF], UL[q]);
    ld_rec<NF, R>(&Uf[(long long)sR[q] * NF], UR[q]);
    ld_nrm<ND, R>(&nrm[(long long)ii[q] * ND], nv[q]);
    aL[q] = dAL[ii[q]];
    aR[q] = dAR[ii[q]];
  }
#pragma unroll
  for (int q = 0; q < PPT; q++) {
    if (i0 + q * stride >= n) break;
    R F[NF];
    if (ND == 2 && roe) {
      roe2d<R>(UL[q], UR[q], nv[q], gam, F);
    } else {
      const R ws = rusanov<ND, R>(UL[q], UR[q], nv[q], gam, F);
      if (waveSp) waveSp[sL[q]] = ws;
    }
    R FL[NF], FR[NF];
#pragma unroll
    for (int k = 0; k < NF; k++) {
      FL[k] = F[k] * aL[q];
      FR[k] = -F[k] * aR[q];
    }
    st_rec<NF, R>(&Fn[(long long)sL[q] * NF], FL);
    st_rec<NF, R>(&Fn[(long long)sR[q] * NF], FR);
  }
}

template <int ND, typename R>
__global__ void k_faces_boundary(int n0, int n, const int *__restrict__ slotL, const int *__restrict__ slotR,
                                 const R *__restrict__ nrm, const R *__restrict__ dAL, const R *__restrict__ Uf,
                                 R *__restrict__ Fn, double *__restrict__ waveSp, Phys ph) {
  pdl_wait();
  pdl_trigger();
  int i = n0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  face_boundary<ND, R>(i, slotL, slotR, nrm, dAL, Uf, Fn, waveSp, ph);
}

// All face points in one launch (small cases, where the launch count
// dominates): interior points first, then boundary points.
template <int ND, typename R>
__global__ void k_faces_all(int nI, int n, const int *__restrict__ slotL, const int *__restrict__ slotR,
                            const R *__restrict__ nrm, const R *__restrict__ dAL, const R *__restrict__ dAR,
                            const R *__restrict__ Uf, R *__restrict__ Fn, double *__restrict__ waveSp, Phys ph) {
  pdl_wait();
  pdl_trigger();
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (i < nI)
    face_interior<ND, R>(i, slotL, slotR, nrm, dAL, dAR, Uf, Fn, waveSp, R(ph.gamma), ND == 2 && ph.riemannType == 1);
  else
    face_boundary<ND, R>(i, slotL, slotR, nrm, dAL, Uf, Fn, waveSp, ph);
}

// Face points of many order groups in one launch: interior points of all
// groups first (work items istart[g] ..), then their boundary points
// (bstart[g] ..); each point as face_interior / face_boundary on its group's
// arrays.
template <int ND, typename R>
__global__ void k_faces_multi(const __grid_constant__ MultiFaceArgsT<R> m, Phys ph) {
  pdl_wait();
  pdl_trigger();
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  const int G = m.nGroups;
  if (w < m.istart[G]) {
    int g = 0;
    while (g + 1 < G && w >= m.istart[g + 1]) g++;
    const FaceTableT<R> &f = m.ft[g];
    face_interior<ND, R>(w - m.istart[g], f.slotL, f.slotR, f.nrm, f.dAL, f.dAR, m.Uf[g], m.Fn[g], m.wave[g],
                         R(ph.gamma), ND == 2 && ph.riemannType == 1);
  } else if (w < m.istart[G] + m.bstart[G]) {
    const int v = w - m.istart[G];
    int g = 0;
    while (g + 1 < G && v >= m.bstart[g + 1]) g++;
    const FaceTableT<R> &f = m.ft[g];
    face_boundary<ND, R>(f.nInterior + v - m.bstart[g], f.slotL, f.slotR, f.nrm, f.dAL, m.Uf[g], m.Fn[g], m.wave[g],
                         ph);
  }
}

// A part of a case split by a partition: the traces at its cut face points,
// packed in its cut order for the peers (send[i] = U_fpts at slot[i]).
template <typename R>
__global__ void k_pack_cut(long long n, int nF, const int *__restrict__ slot, const R *__restrict__ Uf,
                           R *__restrict__ send) {
  pdl_wait();
  pdl_trigger();
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * nF) return;
  const long long i = t / nF;
  const int k = (int)(t - i * nF);
  send[t] = Uf[(long long)slot[i] * nF + k];
}

// Cut face point i: the common flux with this part's element as the left
// side and the peer's trace at the same point as the right state
// (mpiFace::getRightState, src/mpiFace.cpp:158-175, then the interior flux
// of face::calcInviscidFlux, face.cpp:163-208), written to this side only.
// The wave speed goes to this side only where it was the face's left side in
// the whole mesh, as the unsplit face writes it (face.cpp:372).
template <int ND, typename R>
__global__ void k_faces_cut(int n, const int *__restrict__ slot, const int *__restrict__ left,
                            const R *__restrict__ nrm, const R *__restrict__ dA, const R *__restrict__ Uf,
                            const R *__restrict__ recv, R *__restrict__ Fn, double *__restrict__ waveSp, R gam,
                            int roe) {
  pdl_wait();
  pdl_trigger();
  constexpr int NF = ND + 2;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int s = slot[i];
  R UL[NF], UR[NF], nv[ND], F[NF];
#pragma unroll
  for (int k = 0; k < NF; k++) UL[k] = Uf[(long long)s * NF + k];
#pragma unroll
  for (int k = 0; k < NF; k++) UR[k] = recv[(long long)i * NF + k];
#pragma unroll
  for (int d = 0; d < ND; d++) nv[d] = nrm[(long long)i * ND + d];
  if (ND == 2 && roe) {
    roe2d<R>(UL, UR, nv, gam, F);
  } else {
    const R ws = rusanov<ND, R>(UL, UR, nv, gam, F);
    if (waveSp && left[i]) waveSp[s] = ws;
  }
  const R a = dA[i];
#pragma unroll
  for (int k = 0; k < NF; k++) Fn[(long long)s * NF + k] = F[k] * a;
}

// Every device scalar dt[0..n) set to their minimum (the time step of a
// case split into parts, MPI_Allreduce(MIN) in solver::calcDt,
// src/solver.cpp:462-465).
struct DtPtrs {
  double *p[kMaxParts];
};
__global__ void k_min_dt(DtPtrs d, int n) {
  pdl_wait();
  pdl_trigger();
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double m = *d.p[0];
  for (int i = 1; i < n; i++) m = fmin(m, *d.p[i]);
  for (int i = 0; i < n; i++) *d.p[i] = m;
}

__device__ __forceinline__ double csr_dot(const Csr &A, int row, const double *__restrict__ x,
                                          int stride) {
  double s = 0.0;
  const int b = A.rowptr[row], e = A.rowptr[row + 1];
  for (int j = b; j < e; j++) s += A.val[j] * x[A.col[j] * stride];
  return s;
}

template <int ND>
__global__ void __launch_bounds__(256) k_element_stage(ElemArgs a) {
  pdl_wait();
  pdl_trigger();
  constexpr int NF = ND + 2;
  extern __shared__ double smem[];
  const int EB = a.EB, nS = a.nS, nFp = a.nFp, E = a.E;
  const int e0 = blockIdx.x * EB;
  const int nValid = min(EB, E - e0);
  const int rowS = EB * NF;  // doubles per point row of a tile
  double *sU = smem;                      // [nS][EB][NF]
  double *sF = sU + (size_t)nS * rowS;    // [ND][nS][EB][NF]
  double *sQ = sF + (size_t)ND * nS * rowS;  // [nFp][EB][NF]
  double *sD = sQ + (size_t)nFp * rowS;   // [nS][EB][NF]

  // A: stage the state tile (coalesced: each point row is EB*NF contiguous)
  for (int idx = threadIdx.x; idx < nS * rowS; idx += blockDim.x) {
    const int s = idx / rowS, r = idx - s * rowS;
    sU[idx] = (r < nValid * NF) ? a.U[((long long)s * E + e0) * NF + r] : 1.0;
  }
  __syncthreads();

  // B: reference-space flux at the solution points
  for (int it = threadIdx.x; it < nS * EB; it += blockDim.x) {
    const int s = it / EB, el = it - s * EB;
    const int e = e0 + el;
    double Fp[ND][NF];
    const double *u = &sU[(s * EB + el) * NF];
    if (el < nValid) {
      inviscid_flux<ND, double>(u, Fp, a.gamma);
    } else {
#pragma unroll
      for (int d = 0; d < ND; d++)
#pragma unroll
        for (int k = 0; k < NF; k++) Fp[d][k] = 0.0;
    }
#pragma unroll
    for (int d1 = 0; d1 < ND; d1++) {
      double J[ND];
#pragma unroll
      for (int d2 = 0; d2 < ND; d2++)
        J[d2] = el < nValid ? a.JGinv[(((long long)d1 * nS + s) * E + e) * ND + d2] : 0.0;
#pragma unroll
      for (int k = 0; k < NF; k++) {
        double f = 0.0;
#pragma unroll
        for (int d2 = 0; d2 < ND; d2++) f += J[d2] * Fp[d2][k];
        sF[((d1 * nS + s) * EB + el) * NF + k] = f;
        if (a.F_dbg && el < nValid) a.F_dbg[(((long long)d1 * nS + s) * E + e) * NF + k] = f;
      }
    }
  }
  __syncthreads();

  // C: flux divergence at the solution points and (Fn - extrapolated normal
  // flux) at the flux points
  for (int it = threadIdx.x; it < (nS + nFp) * EB; it += blockDim.x) {
    if (it < nS * EB) {
      const int s = it / EB, el = it - s * EB;
#pragma unroll
      for (int k = 0; k < NF; k++) {
        const double *x0 = &sF[el * NF + k];
        double t = csr_dot(a.grad[0], s, x0, rowS);
#pragma unroll
        for (int d = 1; d < ND; d++) t = t + csr_dot(a.grad[d], s, x0 + (size_t)d * nS * rowS, rowS);
        sD[(s * EB + el) * NF + k] = t;
      }
    } else {
      const int j = it - nS * EB;
      const int f = j / EB, el = j - f * EB;
      const int e = e0 + el;
#pragma unroll
      for (int k = 0; k < NF; k++) {
        const double *x0 = &sF[el * NF + k];
        double t = csr_dot(a.extFn[0], f, x0, rowS);
#pragma unroll
        for (int d = 1; d < ND; d++) t = t + csr_dot(a.extFn[d], f, x0 + (size_t)d * nS * rowS, rowS);
        double q = el < nValid ? a.Fn[((long long)f * E + e) * NF + k] - t : 0.0;
        sQ[(f * EB + el) * NF + k] = q;
        if (a.disFn_dbg && el < nValid) a.disFn_dbg[((long long)f * E + e) * NF + k] = q;
      }
    }
  }
  __syncthreads();

  // D: correction, RK update
  const double dtg = (a.mode != MODE_RESIDUAL && a.dt) ? *a.dt : 0.0;
  for (int it = threadIdx.x; it < nS * EB; it += blockDim.x) {
    const int s = it / EB, el = it - s * EB;
    const int e = e0 + el;
    if (el >= nValid) continue;
    const double rdJ = 1.0 / a.detJ[(long long)s * E + e];  // one reciprocal per point
    const double dt = a.eleDt ? a.eleDt[e] : dtg;
#pragma unroll
    for (int k = 0; k < NF; k++) {
      const int li = (s * EB + el) * NF + k;
      const long long gi = ((long long)s * E + e) * NF + k;
      double div = csr_dot(a.corr, s, &sQ[el * NF + k], rowS) + sD[li];
      if (a.divF_out) a.divF_out[gi] = div;
      if (a.mode == MODE_RESIDUAL) continue;
      if (a.src) div = div + a.src[gi];
      const double u = sU[li];
      double unew;
      if (a.mode == MODE_RK_STAGE) {
        const double u0 = a.stage == 0 ? u : a.U0[gi];
        if (a.stage == 0) a.U0[gi] = u;
        unew = u0 - a.rka_next * div * rdJ * dt;
        const double base = a.stage == 0 ? u0 : a.acc[gi];
        a.acc[gi] = base - a.rkb * div * rdJ * dt;
      } else if (a.mode == MODE_RK_FINAL) {
        const double base = a.nRK == 1 ? u : a.acc[gi];
        unew = base - a.rkb * div * rdJ * dt;
      } else {  // MODE_JAMESON
        const double u0 = a.stage == 0 ? u : a.U0[gi];
        if (a.stage == 0) a.U0[gi] = u;
        unew = u0 - a.rka_next * div * rdJ * dt;
      }
      a.Uout[gi] = unew;
      sU[li] = unew;
    }
  }
  if (a.mode == MODE_RESIDUAL || !a.Ufpts_out) return;
  __syncthreads();

  // E: new state at the flux points
  for (int it = threadIdx.x; it < nFp * EB; it += blockDim.x) {
    const int f = it / EB, el = it - f * EB;
    if (el >= nValid) continue;
    const int e = e0 + el;
#pragma unroll
    for (int k = 0; k < NF; k++)
      a.Ufpts_out[((long long)f * E + e) * NF + k] = csr_dot(a.ext, f, &sU[el * NF + k], rowS);
  }
}

// FP64 arithmetic for either state type (the time step stays FP64)
template <int ND, typename R>
__global__ void k_wavesp_init(int nFp, int E, const R *__restrict__ Uf, const double *__restrict__ norm, double gam,
                              double *__restrict__ waveSp) {
  pdl_wait();
  pdl_trigger();
  constexpr int NF = ND + 2;
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)nFp * E) return;
  const R *U = &Uf[i * NF];
  const double *n = &norm[i * ND];
  double rho = U[0];
  double u = U[1] / rho;
  double v = U[2] / rho;
  double w = 0;
  if (ND == 3) w = U[3] / rho;
  double rhoVSq = rho * (u * u + v * v + w * w);
  double p = (gam - 1) * (U[ND + 1] - 0.5 * rhoVSq);
  double vN = u * n[0] + v * n[1];
  if (ND == 3) vN += w * n[ND - 1];
  double csq = fmax(gam * p / rho, 0.0);
  waveSp[i] = fabs(vN - 0.0) + sqrt(csq);
}

__global__ void k_element_dt(int nS, int nFp, int nPF, int E, const double *__restrict__ detJ,
                             const double *__restrict__ wSpt, const double *__restrict__ wSurf,
                             const double *__restrict__ waveSp, const double *__restrict__ dA,
                             double cflFac, double *__restrict__ eleDt,
                             unsigned long long *dtMinBits) {
  pdl_wait();
  pdl_trigger();
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= E) return;
  double vol = 0;
  for (int s = 0; s < nS; s++) vol += detJ[(long long)s * E + e] * wSpt[s];
  double intWave = 0;
  for (int f = 0; f < nFp; f++)
    intWave += waveSp[(long long)f * E + e] * wSurf[f % nPF] * dA[(long long)f * E + e];
  double dt = cflFac * 2 * vol / intWave;
  if (eleDt) eleDt[e] = dt;
  if (dtMinBits && dt >= 0.0 && dt == dt)
    atomicMin(dtMinBits, (unsigned long long)__double_as_longlong(dt));
}

// Element dt and the global minimum in one launch: each block reduces its
// elements' dt (bit patterns of non-negative doubles order like the values)
// and folds it into *bits with atomicMin; the last block to finish stores
// the minimum in *dt and resets *bits and *count for the next call, so no
// separate reset or store launch is needed (*bits must start at +inf and
// *count at 0).
__global__ void k_element_dt_min(int nS, int nFp, int nPF, int E, const double *__restrict__ detJ,
                                 const double *__restrict__ wSpt, const double *__restrict__ wSurf,
                                 const double *__restrict__ waveSp, const double *__restrict__ dA, double cflFac,
                                 double *__restrict__ eleDt, unsigned long long *bits, unsigned int *count,
                                 double *dtOut) {
  pdl_wait();
  pdl_trigger();
  __shared__ unsigned long long sMin[32];
  __shared__ bool last;
  const unsigned long long INF = (unsigned long long)0x7ff0000000000000ull;
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long mine = INF;
  if (e < E) {
    double vol = 0;
    for (int s = 0; s < nS; s++) vol += detJ[(long long)s * E + e] * wSpt[s];
    double intWave = 0;
    for (int f = 0; f < nFp; f++)
      intWave += waveSp[(long long)f * E + e] * wSurf[f % nPF] * dA[(long long)f * E + e];
    double dt = cflFac * 2 * vol / intWave;
    if (eleDt) eleDt[e] = dt;
    if (dt >= 0.0 && dt == dt) mine = (unsigned long long)__double_as_longlong(dt);
  }
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long v = __shfl_xor_sync(0xffffffffu, mine, o);
    mine = v < mine ? v : mine;
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) sMin[w] = mine;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long m = INF;
    for (int i = 0; i < (int)((blockDim.x + 31) / 32); i++) m = sMin[i] < m ? sMin[i] : m;
    if (m != INF) atomicMin(bits, m);
    __threadfence();
    last = atomicAdd(count, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (last && threadIdx.x == 0) {
    __threadfence();
    const unsigned long long m = atomicAdd(bits, 0ull);
    *dtOut = __longlong_as_double((long long)m);
    *bits = INF;
    *count = 0;
  }
}

__global__ void k_reset_min(unsigned long long *bits) {
  pdl_wait();
  pdl_trigger();
  *bits = (unsigned long long)__double_as_longlong(__longlong_as_double(0x7ff0000000000000ll));
}

__global__ void k_store_min(const unsigned long long *bits, double *dt, double *time_acc) {
  pdl_wait();
  pdl_trigger();
  *dt = __longlong_as_double((long long)*bits);
  (void)time_acc;
}

__global__ void k_add_time(const double *dt, double *time_acc) {
  pdl_wait();
  pdl_trigger(); *time_acc += *dt; }

template <typename R>
__global__ void k_residual_norm(int nS, int E, int nF, const R *__restrict__ divF, const double *__restrict__ detJ,
                                const double *__restrict__ w, int resType, double *__restrict__ eleRes) {
  pdl_wait();
  pdl_trigger();
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= E) return;
  for (int k = 0; k < nF; k++) {
    double r = 0;
    for (int s = 0; s < nS; s++) {
      double d = divF[((long long)s * E + e) * nF + k];
      if (resType == 1)
        r += fabs(d) * w[s];
      else if (resType == 2)
        r += d * d / detJ[(long long)s * E + e] * w[s];
      else  // a NaN anywhere makes the maximum NaN (fmax would drop it)
        r = nan_max(fabs(d) / detJ[(long long)s * E + e], r);
    }
    eleRes[(long long)e * nF + k] = r;
  }
}

template <typename R>
__global__ void k_add(long long n, R *__restrict__ out, const R *__restrict__ x, const R *__restrict__ y, double sgn) {
  pdl_wait();
  pdl_trigger();
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  out[i] = sgn > 0 ? x[i] + y[i] : x[i] - y[i];
}

template <typename R>
__global__ void k_check_state(long long n, int nF, const R *__restrict__ U, unsigned int *bad) {
  pdl_wait();
  pdl_trigger();
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  R v = U[i];
  bool b = !(v == v) || isinf(v);
  if ((i % nF) == 0 && !(v > R(0))) b = true;
  if (b) atomicAdd(bad, 1u);
}

template <typename R>
__global__ void k_apply_op_t(int nRows, const int *__restrict__ rp, const int *__restrict__ ci,
                             const double *__restrict__ v, const R *__restrict__ in, R *__restrict__ out, long long N) {
  pdl_wait();
  pdl_trigger();
  long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  int r = blockIdx.y;
  if (n >= N || r >= nRows) return;
  R s = R(0);
  for (int j = rp[r]; j < rp[r + 1]; j++) s += R(v[j]) * in[(long long)ci[j] * N + n];
  out[(long long)r * N + n] = s;
}

__global__ void k_split(long long n, const double *__restrict__ U64, float *__restrict__ U32,
                        float *__restrict__ comp) {
  pdl_wait();
  pdl_trigger();
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double u = U64[i];
  const float hi = __double2float_rn(u);
  U32[i] = hi;
  comp[i] = __double2float_rn(u - (double)hi);
}

__global__ void k_join(long long n, const float *__restrict__ U32, const float *__restrict__ comp,
                       double *__restrict__ U64) {
  pdl_wait();
  pdl_trigger();
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  U64[i] = (double)U32[i] + (double)comp[i];
}

__global__ void k_narrow(long long n, const double *__restrict__ in, float *__restrict__ out) {
  pdl_wait();
  pdl_trigger();
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = __double2float_rn(in[i]);
}

__global__ void k_widen(long long n, const float *__restrict__ in, double *__restrict__ out) {
  pdl_wait();
  pdl_trigger();
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = (double)in[i];
}

}  // namespace

void launch_apply_op(const Csr &A, const double *in, double *out, long long N, double alpha,
                     double beta, cudaStream_t st) {
  if (N <= 0 || A.nRows <= 0) return;
  dim3 g((unsigned)((N + 255) / 256), (unsigned)A.nRows);
  launch_k(k_apply_op, g, 256, 0, st, A.nRows, A.rowptr, A.col, A.val, in, out, N, alpha, beta);
}

template <typename R>
void launch_apply_op_t(const Csr &A, const R *in, R *out, long long N, cudaStream_t st) {
  if (N <= 0 || A.nRows <= 0) return;
  dim3 g((unsigned)((N + 255) / 256), (unsigned)A.nRows);
  launch_k(k_apply_op_t<R>, g, 256, 0, st, A.nRows, A.rowptr, A.col, A.val, in, out, N);
}

template <typename R>
void launch_faces_inviscid(int nDims, const FaceTableT<R> &ft, const R *Ufpts, R *Fn, double *waveSp,
                           const Phys &ph, cudaStream_t st) {
  const int b = 256;
  const int nI = ft.nInterior, nB = ft.n - ft.nInterior;
  if (nI > 0 && nB > 0 && pdl_enabled()) {  // small case: one launch
    const int g = (ft.n + b - 1) / b;
    if (nDims == 2)
      launch_k(k_faces_all<2, R>, g, b, 0, st, nI, ft.n, ft.slotL, ft.slotR, ft.nrm, ft.dAL, ft.dAR, Ufpts, Fn,
               waveSp, ph);
    else
      launch_k(k_faces_all<3, R>, g, b, 0, st, nI, ft.n, ft.slotL, ft.slotR, ft.nrm, ft.dAL, ft.dAR, Ufpts, Fn,
               waveSp, ph);
    return;
  }
  if (nI > 0) {
    // two points per thread (2-D FP32 with the vector record accesses:
    // vortex 512^2 P3 face pass 0.0412 -> 0.0350 ms against one point per
    // thread; with per-value accesses one point per thread had been faster)
    const int per = kFaceNt * kFacePpt;
    const int g = (nI + per - 1) / per;
    if (nDims == 2)
      launch_k(k_faces_interior_ilp<2, R, kFacePpt>, g, kFaceNt, 0, st, nI, ft.slotL, ft.slotR, ft.nrm, ft.dAL,
               ft.dAR, Ufpts, Fn, waveSp, R(ph.gamma), ph.riemannType == 1);
    else
      launch_k(k_faces_interior_ilp<3, R, kFacePpt>, g, kFaceNt, 0, st, nI, ft.slotL, ft.slotR, ft.nrm, ft.dAL,
               ft.dAR, Ufpts, Fn, waveSp, R(ph.gamma), 0);
  }
  if (nB > 0) {
    const int g = (nB + b - 1) / b;
    if (nDims == 2)
      launch_k(k_faces_boundary<2, R>, g, b, 0, st, nI, ft.n, ft.slotL, ft.slotR, ft.nrm, ft.dAL, Ufpts, Fn, waveSp, ph);
    else
      launch_k(k_faces_boundary<3, R>, g, b, 0, st, nI, ft.n, ft.slotL, ft.slotR, ft.nrm, ft.dAL, Ufpts, Fn, waveSp, ph);
  }
}

size_t elem_smem_bytes(int nDims, int nS, int nFp, int EB) {
  int nF = nDims + 2;
  return sizeof(double) * (size_t)EB * nF * ((size_t)nS * (2 + nDims) + nFp);
}

void launch_element_stage(int nDims, const ElemArgs &a, cudaStream_t st) {
  if (a.E <= 0) return;
  int g = (a.E + a.EB - 1) / a.EB;
  size_t sm = elem_smem_bytes(nDims, a.nS, a.nFp, a.EB);
  if (nDims == 2) {
    cudaFuncSetAttribute(k_element_stage<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    launch_k(k_element_stage<2>, g, 256, sm, st, a);
  } else {
    cudaFuncSetAttribute(k_element_stage<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    launch_k(k_element_stage<3>, g, 256, sm, st, a);
  }
}

template <typename R>
void launch_wavesp_init(int nDims, int nFp, int E, const R *Ufpts, const double *norm, double gamma,
                        double *waveSp, cudaStream_t st) {
  long long n = (long long)nFp * E;
  if (n <= 0) return;
  unsigned g = (unsigned)((n + 255) / 256);
  if (nDims == 2)
    launch_k(k_wavesp_init<2, R>, g, 256, 0, st, nFp, E, Ufpts, norm, gamma, waveSp);
  else
    launch_k(k_wavesp_init<3, R>, g, 256, 0, st, nFp, E, Ufpts, norm, gamma, waveSp);
}

void launch_element_dt(int nDims, int nS, int nFp, int nPF, int E, const double *detJ,
                       const double *wSpt, const double *wSurf, const double *waveSp,
                       const double *dA, double cflFac, double *eleDt,
                       unsigned long long *dtMinBits, cudaStream_t st) {
  (void)nDims;
  if (E <= 0) return;
  launch_k(k_element_dt, (E + 127) / 128, 128, 0, st, nS, nFp, nPF, E, detJ, wSpt, wSurf, waveSp, dA,
                                                 cflFac, eleDt, dtMinBits);
}

void launch_element_dt_min(int nS, int nFp, int nPF, int E, const double *detJ, const double *wSpt,
                           const double *wSurf, const double *waveSp, const double *dA, double cflFac, double *eleDt,
                           unsigned long long *bits, unsigned int *count, double *dt, cudaStream_t st) {
  if (E <= 0) return;
  launch_k(k_element_dt_min, (E + 127) / 128, 128, 0, st, nS, nFp, nPF, E, detJ, wSpt, wSurf, waveSp, dA, cflFac,
           eleDt, bits, count, dt);
}

void launch_reset_min(unsigned long long *bits, cudaStream_t st) { launch_k(k_reset_min, 1, 1, 0, st, bits); }

void launch_store_min(const unsigned long long *bits, double *dt, double *time_acc, cudaStream_t st) {
  launch_k(k_store_min, 1, 1, 0, st, bits, dt, time_acc);
}

void launch_add_time(const double *dt, double *time_acc, cudaStream_t st) {
  launch_k(k_add_time, 1, 1, 0, st, dt, time_acc);
}

template <typename R>
void launch_residual_norm(int nS, int E, int nF, const R *divF, const double *detJ, const double *wSpt,
                          int resType, double *eleRes, cudaStream_t st) {
  if (E <= 0) return;
  launch_k(k_residual_norm<R>, (E + 127) / 128, 128, 0, st, nS, E, nF, divF, detJ, wSpt, resType, eleRes);
}

void launch_add(long long n, double *out, const double *x, const double *y, double sgn, cudaStream_t st) {
  if (n <= 0) return;
  launch_k(k_add<double>, (unsigned)((n + 255) / 256), 256, 0, st, n, out, x, y, sgn);
}

void launch_add32(long long n, float *out, const float *x, const float *y, double sgn, cudaStream_t st) {
  if (n <= 0) return;
  launch_k(k_add<float>, (unsigned)((n + 255) / 256), 256, 0, st, n, out, x, y, sgn);
}

template <typename R>
void launch_check_state(int nS, int E, int nF, const R *U, unsigned int *bad, cudaStream_t st) {
  long long n = (long long)nS * E * nF;
  if (n <= 0) return;
  launch_k(k_check_state<R>, (unsigned)((n + 255) / 256), 256, 0, st, n, nF, U, bad);
}

void launch_split(long long n, const double *U64, float *U32, float *comp, cudaStream_t st) {
  if (n > 0) launch_k(k_split, (unsigned)((n + 255) / 256), 256, 0, st, n, U64, U32, comp);
}
void launch_join(long long n, const float *U32, const float *comp, double *U64, cudaStream_t st) {
  if (n > 0) launch_k(k_join, (unsigned)((n + 255) / 256), 256, 0, st, n, U32, comp, U64);
}
void launch_narrow(long long n, const double *in, float *out, cudaStream_t st) {
  if (n > 0) launch_k(k_narrow, (unsigned)((n + 255) / 256), 256, 0, st, n, in, out);
}
void launch_widen(long long n, const float *in, double *out, cudaStream_t st) {
  if (n > 0) launch_k(k_widen, (unsigned)((n + 255) / 256), 256, 0, st, n, in, out);
}

template <typename R>
void launch_faces_multi(int nDims, const MultiFaceArgsT<R> &m, const Phys &ph, cudaStream_t st) {
  const int n = m.istart[m.nGroups] + m.bstart[m.nGroups];
  if (n <= 0) return;
  const int b = 128, g = (n + b - 1) / b;
  if (nDims == 2)
    launch_k(k_faces_multi<2, R>, g, b, 0, st, m, ph);
  else
    launch_k(k_faces_multi<3, R>, g, b, 0, st, m, ph);
}

template <typename R>
void launch_pack_cut(int nF, const CutTableT<R> &c, const R *Ufpts, cudaStream_t st) {
  const long long n = (long long)c.n * nF;
  if (n > 0) launch_k(k_pack_cut<R>, (unsigned)((n + 255) / 256), 256, 0, st, (long long)c.n, nF, c.slot, Ufpts, c.send);
}

template <typename R>
void launch_faces_cut(int nDims, const CutTableT<R> &c, const R *Ufpts, R *Fn, double *waveSp, const Phys &ph,
                      cudaStream_t st) {
  if (c.n <= 0) return;
  const int b = 128, g = (c.n + b - 1) / b;
  if (nDims == 2)
    launch_k(k_faces_cut<2, R>, g, b, 0, st, c.n, c.slot, c.left, c.nrm, c.dA, Ufpts, c.recv, Fn, waveSp,
             R(ph.gamma), ph.riemannType == 1);
  else
    launch_k(k_faces_cut<3, R>, g, b, 0, st, c.n, c.slot, c.left, c.nrm, c.dA, Ufpts, c.recv, Fn, waveSp,
             R(ph.gamma), 0);
}

void launch_min_dt(double *const *dts, int n, cudaStream_t st) {
  if (n <= 1) return;
  DtPtrs d{};
  for (int i = 0; i < n && i < kMaxParts; i++) d.p[i] = dts[i];
  launch_k(k_min_dt, 1, 32, 0, st, d, n < kMaxParts ? n : kMaxParts);
}

#define FR_BASE_INST(R)                                                                                        \
  template void launch_apply_op_t<R>(const Csr &, const R *, R *, long long, cudaStream_t);                   \
  template void launch_faces_inviscid<R>(int, const FaceTableT<R> &, const R *, R *, double *, const Phys &,  \
                                         cudaStream_t);                                                       \
  template void launch_wavesp_init<R>(int, int, int, const R *, const double *, double, double *, cudaStream_t); \
  template void launch_residual_norm<R>(int, int, int, const R *, const double *, const double *, int, double *, \
                                        cudaStream_t);                                                        \
  template void launch_check_state<R>(int, int, int, const R *, unsigned int *, cudaStream_t);               \
  template void launch_pack_cut<R>(int, const CutTableT<R> &, const R *, cudaStream_t);                     \
  template void launch_faces_multi<R>(int, const MultiFaceArgsT<R> &, const Phys &, cudaStream_t);          \
  template void launch_faces_cut<R>(int, const CutTableT<R> &, const R *, R *, double *, const Phys &,      \
                                    cudaStream_t);
FR_BASE_INST(double)
FR_BASE_INST(float)
#undef FR_BASE_INST

}  // namespace frk
