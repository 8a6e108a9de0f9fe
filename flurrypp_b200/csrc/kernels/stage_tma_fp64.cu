// Tensor-product element kernel, FP64, with TMA tile transfers.
//
// The same stage as k_elem_tp (reference: solver.cpp:470-572, 707-736,
// 906-1058), but each CTA fetches all of its input tiles at once with
// cp.async.bulk.tensor loads completing on one mbarrier (state U, the RK base
// U0 and running sum acc, metrics JGinv and detJ, common flux Fn), and writes
// U, acc, U0 and U_fpts back with cp.async.bulk.tensor stores.  A tile is one
// operator row block [points][EB elements x fields], which is contiguous in
// the reference layout, so every transfer is one TMA instruction.
//
// Requirements (checked on the host): E*nFields and E*nDims even (16-byte
// row pitch) and the element block EB even (16-byte aligned x offsets).
#include "stage.hpp"
#include "tma.cuh"

namespace frk {

namespace {

constexpr int ipow2(int b, int e) { return e == 0 ? 1 : b * ipow2(b, e - 1); }

template <int ND, int P>
struct Tm {
  static constexpr int N = P + 1;
  static constexpr int NF = ND + 2;
  static constexpr int NS = ipow2(N, ND);
  static constexpr int NPF = ipow2(N, ND - 1);
  static constexpr int NFP = 2 * ND * NPF;
  // largest power of two <= 32 with NS*EB <= 160, at least 2
  static constexpr int EB = NS * 32 <= 160 ? 32 : NS * 16 <= 160 ? 16 : NS * 8 <= 160 ? 8 : NS * 4 <= 160 ? 4 : 2;
  static constexpr int NT = NS * EB;
  static constexpr int ROW = EB * NF;
  // shared-memory carve-up, in doubles; every tile starts on 128 bytes
  static constexpr int al(int n) { return (n + 15) / 16 * 16; }
  static constexpr int O_U = 0;
  static constexpr int O_U0 = O_U + al(NS * ROW);
  static constexpr int O_ACC = O_U0 + al(NS * ROW);
  static constexpr int O_FN = O_ACC + al(NS * ROW);
  static constexpr int O_J = O_FN + al(NFP * ROW);
  static constexpr int O_DET = O_J + al(ND * NS * EB * ND);
  static constexpr int O_F = O_DET + al(NS * EB);
  static constexpr int O_TAB = O_F + al(ND * NS * ROW);
  static constexpr int O_CV = O_TAB + al(N * N + 4 * N);       // corrVal [NS][2ND] doubles
  static constexpr int O_IDX = O_CV + al(NS * 2 * ND);          // ints: fpt line [NFP], corrFpt [NS][2ND]
  static constexpr int O_BAR = O_IDX + al((NFP + NS * 2 * ND + 1) / 2);
  static constexpr size_t SMEM = sizeof(double) * (size_t)(O_BAR + 4) + 128;
};

template <int ND, int P>
__global__ void __launch_bounds__(Tm<ND, P>::NT) k_elem_tma(ElemArgs a, TpTables t,
                                                            const __grid_constant__ TmaMaps mp) {
  using T = Tm<ND, P>;
  constexpr int N = T::N, NF = T::NF, NS = T::NS, NFP = T::NFP, EB = T::EB, NT = T::NT, ROW = T::ROW;
  extern __shared__ __align__(128) double smem_raw[];
  // tiles start on 128-byte boundaries relative to an aligned base
  double *smem = reinterpret_cast<double *>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
  double *sU = smem + T::O_U;
  double *sU0 = smem + T::O_U0;
  double *sAcc = smem + T::O_ACC;
  double *sFn = smem + T::O_FN;   // Fn -> Fn - extrapolated flux -> new U_fpts
  double *sJ = smem + T::O_J;     // [ND][NS][EB*ND]
  double *sDet = smem + T::O_DET; // [NS][EB]
  double *sF = smem + T::O_F;     // [ND][NS][ROW]
  double *sD = smem + T::O_TAB;
  double *sE = sD + N * N;
  double *sEF = sE + 2 * N;
  double *sCV = smem + T::O_CV;
  int *sLine = reinterpret_cast<int *>(smem + T::O_IDX);  // base | dn << 16 | side << 20
  int *sCF = sLine + NFP;
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem + T::O_BAR);

  const int E = a.E;
  const int e0 = blockIdx.x * EB;
  const int nValid = min(EB, E - e0);
  const int tid = threadIdx.x;
  const int s = tid / EB, el = tid - (tid / EB) * EB;
  const int e = e0 + el;
  const bool valid = el < nValid;

  const bool needU0 = (a.mode == MODE_RK_STAGE || a.mode == MODE_JAMESON) && a.stage > 0;
  const bool needAcc = (a.mode == MODE_RK_STAGE && a.stage > 0) || (a.mode == MODE_RK_FINAL && a.nRK > 1);
  const bool needDet = a.mode != MODE_RESIDUAL;

  // two transaction barriers: bar[0] for what the flux needs (U, JGinv),
  // bar[1] for what the correction and update need (Fn, U0, acc, detJ), so
  // the second batch lands while the flux and divergence are computed
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (tid == 0) {
    mbar_arrive_expect_tx(&bar[0], sizeof(double) * (NS * ROW + ND * NS * EB * ND));
    tma_load_2d(sU, &mp.U, e0 * NF, 0, &bar[0]);
    tma_load_3d(sJ, &mp.J, e0 * ND, 0, 0, &bar[0]);
    uint32_t bytes = sizeof(double) * NFP * ROW;
    if (needU0) bytes += sizeof(double) * NS * ROW;
    if (needAcc) bytes += sizeof(double) * NS * ROW;
    if (needDet) bytes += sizeof(double) * NS * EB;
    mbar_arrive_expect_tx(&bar[1], bytes);
    tma_load_2d(sFn, &mp.Fn, e0 * NF, 0, &bar[1]);
    if (needU0) tma_load_2d(sU0, &mp.U0, e0 * NF, 0, &bar[1]);
    if (needAcc) tma_load_2d(sAcc, &mp.acc, e0 * NF, 0, &bar[1]);
    if (needDet) tma_load_2d(sDet, &mp.det, e0, 0, &bar[1]);
  }
  for (int i = tid; i < N * N; i += NT) sD[i] = t.D[i];
  for (int i = tid; i < 2 * N; i += NT) {
    sE[i] = t.E1[i];
    sEF[i] = t.EFn1[i];
  }
  for (int i = tid; i < NFP; i += NT) sLine[i] = t.fptBase[i] | (t.fptDn[i] << 16) | (t.fptSide[i] << 20);
  for (int i = tid; i < NS * 2 * ND; i += NT) {
    sCF[i] = t.corrFpt[i];
    sCV[i] = t.corrVal[i];
  }
  if (!mbar_wait_bounded(&bar[0], 0, 1u << 22)) {
    // give up: flag it, let the copies in flight land (bounded), leave
    if (a.err) atomicOr(a.err, 1);
    mbar_wait_bounded(&bar[0], 0, 1u << 22);
    mbar_wait_bounded(&bar[1], 0, 1u << 22);
    return;
  }
  __syncthreads();  // tables

  // stage 0: the RK base state is the state at the start of the step
  if ((a.mode == MODE_RK_STAGE || a.mode == MODE_JAMESON) && a.stage == 0 && tid == 0) {
    tma_store_2d(&mp.U0, e0 * NF, 0, sU);
    tma_commit();
  }

  // B: reference-space flux at (s, el)
  {
    double Fp[ND][NF];
    const double *u = &sU[s * ROW + el * NF];
    if (valid) {
      inviscid_flux<ND, double>(u, Fp, a.gamma);
    } else {
#pragma unroll
      for (int d = 0; d < ND; d++)
#pragma unroll
        for (int k = 0; k < NF; k++) Fp[d][k] = 0.0;
    }
#pragma unroll
    for (int d1 = 0; d1 < ND; d1++) {
      const double *Jr = &sJ[(d1 * NS + s) * EB * ND + el * ND];
#pragma unroll
      for (int k = 0; k < NF; k++) {
        double f = 0.0;
#pragma unroll
        for (int d2 = 0; d2 < ND; d2++) f += Jr[d2] * Fp[d2][k];
        sF[(d1 * NS + s) * ROW + el * NF + k] = f;
        if (a.F_dbg && valid) a.F_dbg[(((long long)d1 * NS + s) * E + e) * NF + k] = f;
      }
    }
  }
  __syncthreads();

  // C1: flux divergence at (s, el)
  int idx3[3];
  idx3[0] = s % N;
  idx3[1] = ND > 1 ? (s / N) % N : 0;
  idx3[2] = ND > 2 ? s / (N * N) : 0;
  double div[NF];
#pragma unroll
  for (int d = 0; d < ND; d++) {
    const int stride = d == 0 ? 1 : (d == 1 ? N : N * N);
    const int base = s - idx3[d] * stride;
    const double *Dr = &sD[idx3[d] * N];
    double acc[NF];
#pragma unroll
    for (int k = 0; k < NF; k++) acc[k] = 0.0;
#pragma unroll
    for (int m = 0; m < N; m++) {
      const double dv = Dr[m];
      const double *x = &sF[(d * NS + base + m * stride) * ROW + el * NF];
#pragma unroll
      for (int k = 0; k < NF; k++) acc[k] += dv * x[k];
    }
#pragma unroll
    for (int k = 0; k < NF; k++) div[k] = d == 0 ? acc[k] : div[k] + acc[k];
  }

  if (!mbar_wait_bounded(&bar[1], 0, 1u << 22)) {
    if (a.err) atomicOr(a.err, 1);
    mbar_wait_bounded(&bar[1], 0, 1u << 22);
    if (tid == 0) tma_wait_read_all();
    return;
  }

  // C2: Fn - extrapolated normal flux, in place in the Fn tile
  for (int it = tid; it < NFP * EB; it += NT) {
    const int f = it / EB, fe = it - (it / EB) * EB;
    const int ln = sLine[f];
    const int base = ln & 0xffff, dn = (ln >> 16) & 0xf, side = ln >> 20;
    const int stride = dn == 0 ? 1 : (dn == 1 ? N : N * N);
    double acc[NF];
#pragma unroll
    for (int k = 0; k < NF; k++) acc[k] = 0.0;
#pragma unroll
    for (int m = 0; m < N; m++) {
      const double ev = sEF[side * N + m];
      const double *x = &sF[(dn * NS + base + m * stride) * ROW + fe * NF];
#pragma unroll
      for (int k = 0; k < NF; k++) acc[k] += ev * x[k];
    }
    double *q = &sFn[f * ROW + fe * NF];
#pragma unroll
    for (int k = 0; k < NF; k++) {
      q[k] = q[k] - acc[k];
      if (a.disFn_dbg && fe < nValid) a.disFn_dbg[((long long)f * E + e0 + fe) * NF + k] = q[k];
    }
  }
  if (tid == 0) tma_wait_read_all();  // the U0 store has read sU
  __syncthreads();

  // D: correction and RK update at (s, el), in place in sU / sAcc
  {
    double cq[NF];
#pragma unroll
    for (int k = 0; k < NF; k++) cq[k] = 0.0;
#pragma unroll
    for (int fc = 0; fc < 2 * ND; fc++) {
      const int fp = sCF[s * 2 * ND + fc];
      const double cv = sCV[s * 2 * ND + fc];
      const double *x = &sFn[fp * ROW + el * NF];
#pragma unroll
      for (int k = 0; k < NF; k++) cq[k] += cv * x[k];
    }
    // one reciprocal per point instead of a division per update term
    const double rdJ = needDet ? 1.0 / sDet[s * EB + el] : 1.0;
    const double dt = a.mode == MODE_RESIDUAL ? 0.0 : (a.eleDt ? (valid ? a.eleDt[e] : 0.0) : *a.dt);
#pragma unroll
    for (int k = 0; k < NF; k++) {
      const int li = s * ROW + el * NF + k;
      const long long gi = ((long long)s * E + e) * NF + k;
      double dv = cq[k] + div[k];
      if (a.divF_out && valid) a.divF_out[gi] = dv;
      if (a.mode == MODE_RESIDUAL) continue;
      if (a.src && valid) dv = dv + a.src[gi];
      const double u = sU[li];
      double unew;
      if (a.mode == MODE_RK_STAGE) {
        const double u0 = a.stage == 0 ? u : sU0[li];
        unew = u0 - a.rka_next * dv * rdJ * dt;
        const double base = a.stage == 0 ? u0 : sAcc[li];
        sAcc[li] = base - a.rkb * dv * rdJ * dt;
      } else if (a.mode == MODE_RK_FINAL) {
        const double base = a.nRK == 1 ? u : sAcc[li];
        unew = base - a.rkb * dv * rdJ * dt;
      } else {
        const double u0 = a.stage == 0 ? u : sU0[li];
        unew = u0 - a.rka_next * dv * rdJ * dt;
      }
      sU[li] = unew;
    }
  }
  if (a.mode == MODE_RESIDUAL) return;
  fence_async_smem();
  __syncthreads();
  if (tid == 0) {
    tma_store_2d(&mp.U, e0 * NF, 0, sU);
    if (a.mode == MODE_RK_STAGE) tma_store_2d(&mp.acc, e0 * NF, 0, sAcc);
    tma_commit();
  }
  if (!a.Ufpts_out) {
    if (tid == 0) tma_wait_read_all();
    return;
  }

  // E: new state at the flux points, into the Fn tile
  for (int it = tid; it < NFP * EB; it += NT) {
    const int f = it / EB, fe = it - (it / EB) * EB;
    const int ln = sLine[f];
    const int base = ln & 0xffff, dn = (ln >> 16) & 0xf, side = ln >> 20;
    const int stride = dn == 0 ? 1 : (dn == 1 ? N : N * N);
    double acc[NF];
#pragma unroll
    for (int k = 0; k < NF; k++) acc[k] = 0.0;
#pragma unroll
    for (int m = 0; m < N; m++) {
      const double ev = sE[side * N + m];
      const double *x = &sU[(base + m * stride) * ROW + fe * NF];
#pragma unroll
      for (int k = 0; k < NF; k++) acc[k] += ev * x[k];
    }
    double *o = &sFn[f * ROW + fe * NF];
#pragma unroll
    for (int k = 0; k < NF; k++) o[k] = acc[k];
  }
  fence_async_smem();
  __syncthreads();
  if (tid == 0) {
    tma_store_2d(&mp.Ufpts, e0 * NF, 0, sFn);
    tma_commit();
    tma_wait_read_all();
  }
}

template <int ND, int P>
void launch_tma(const ElemArgs &a, const TpTables &t, const TmaMaps &m, cudaStream_t st) {
  using T = Tm<ND, P>;
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_elem_tma<ND, P>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)T::SMEM);
    attr = true;
  }
  int g = (a.E + T::EB - 1) / T::EB;
  k_elem_tma<ND, P><<<g, T::NT, T::SMEM, st>>>(a, t, m);
}

}  // namespace

int tma_elems_per_block(int nDims, int order) {
#define FR_TM_EB(ND, P) \
  if (nDims == ND && order == P) return Tm<ND, P>::EB;
  FR_TM_EB(2, 0) FR_TM_EB(2, 1) FR_TM_EB(2, 2) FR_TM_EB(2, 3) FR_TM_EB(2, 4) FR_TM_EB(2, 5)
  FR_TM_EB(3, 0) FR_TM_EB(3, 1) FR_TM_EB(3, 2) FR_TM_EB(3, 3) FR_TM_EB(3, 4) FR_TM_EB(3, 5)
#undef FR_TM_EB
  return 0;
}

size_t tma_smem_bytes(int nDims, int order) {
#define FR_TM_SM(ND, P) \
  if (nDims == ND && order == P) return Tm<ND, P>::SMEM;
  FR_TM_SM(2, 0) FR_TM_SM(2, 1) FR_TM_SM(2, 2) FR_TM_SM(2, 3) FR_TM_SM(2, 4) FR_TM_SM(2, 5)
  FR_TM_SM(3, 0) FR_TM_SM(3, 1) FR_TM_SM(3, 2) FR_TM_SM(3, 3) FR_TM_SM(3, 4) FR_TM_SM(3, 5)
#undef FR_TM_SM
  return 0;
}

void launch_element_stage_tma(int nDims, int order, const ElemArgs &a, const TpTables &t, const TmaMaps &m,
                              cudaStream_t st) {
  if (a.E <= 0) return;
#define FR_TM_CASE(ND, P) \
  if (nDims == ND && order == P) return launch_tma<ND, P>(a, t, m, st);
  FR_TM_CASE(2, 0) FR_TM_CASE(2, 1) FR_TM_CASE(2, 2) FR_TM_CASE(2, 3) FR_TM_CASE(2, 4) FR_TM_CASE(2, 5)
  FR_TM_CASE(3, 0) FR_TM_CASE(3, 1) FR_TM_CASE(3, 2) FR_TM_CASE(3, 3) FR_TM_CASE(3, 4) FR_TM_CASE(3, 5)
#undef FR_TM_CASE
}

}  // namespace frk
