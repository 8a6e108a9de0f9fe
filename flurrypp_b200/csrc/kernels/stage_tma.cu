// Tensor-product element kernel with TMA tile transfers, FP64 plain form and
// FP32 precision form.
//
// The same stage as k_elem_tp (reference: solver.cpp:470-572, 707-736,
// 906-1058), but each CTA fetches all of its input tiles with
// cp.async.bulk.tensor loads completing on two mbarriers (state U and the
// metrics JGinv first; then the common flux Fn, the RK base U0, the running
// sum acc, detJ and, precision form, the state's rounding remainder comp), and
// writes U, acc, U0, comp and U_fpts back with cp.async.bulk.tensor stores.
// A tile is one operator row block [points][EB elements x fields], which is
// contiguous in the reference layout, so every transfer is one TMA
// instruction.
//
// Requirements (checked on the host): every x offset and row pitch a
// multiple of 16 bytes, i.e. for FP64 E and EB even, for FP32 E and EB
// multiples of 4.
#include <type_traits>

#include "launch.cuh"
#include "stage.hpp"
#include "tma.cuh"

namespace frk {

namespace {

constexpr int ipow2(int b, int e) { return e == 0 ? 1 : b * ipow2(b, e - 1); }
constexpr int pow2_floor(int x) { return x >= 2 ? 2 * pow2_floor(x / 2) : 1; }

constexpr int kFp32Variants = 3;
constexpr int kFp64Variants = 2;
constexpr size_t kMaxSmem = 227 * 1024;

template <int ND, int P, typename R, int V, bool VS = false>
struct Tm {
  static constexpr bool F32 = std::is_same<R, float>::value;
  // FP64 inviscid stages use the lean tile set: the RK base state U0 is read
  // from global memory at each thread's own point (it is read once, so a
  // tile buys nothing) and the flux tile is laid over the metric tile, which
  // every thread copies to registers first.  At 3-D P3 this takes a 2-element
  // CTA from 54.8 to 40.8 KB (36.3 KB with the correction tables below: six
  // CTAs per SM instead of four).  Viscous stages load the gradient into the
  // flux tile together with the metrics.  (smem_for, which only sizes EB,
  // counts the full set.)
  static constexpr bool LEAN = !F32 && !VS;
  static constexpr int N = P + 1;
  static constexpr int NF = ND + 2;
  static constexpr int NS = ipow2(N, ND);
  static constexpr int NPF = ipow2(N, ND - 1);
  static constexpr int NFP = 2 * ND * NPF;
  // in elements of R; every tile starts on 128 bytes
  static constexpr int AL = 128 / (int)sizeof(R);
  static constexpr int al(int n) { return (n + AL - 1) / AL * AL; }
  // FP64 3-D P3: the flux tile is padded by PADR values after each row of N
  // points and PADP after each plane of N*N points.  Unpadded, the plane
  // stride (16 points of EB*NF doubles) is a multiple of 128 bytes, so the
  // lines that end on one face of a hex land 8 deep on the same two banks,
  // and x-lines two deep; padded, every line pattern of the kernel is within
  // one wavefront of conflict-free.  (FP32 tiles, measured, gain nothing.)
  static constexpr bool PADDED = ND == 3 && P == 3 && !F32;
  static constexpr int PADR = PADDED ? 4 : 0, PADP = PADDED ? 2 : 0;
  static constexpr int padF() { return ND == 3 ? N * N * PADR + N * PADP : 0; }
  static constexpr size_t smem_for(int eb) {
    // U, U0, acc, comp tiles; Fn; J; det; F; tables; indices; barriers
    return sizeof(R) * (size_t)(4 * al(NS * eb * NF) + al(NFP * eb * NF) + al(ND * NS * eb * ND) + al(NS * eb) +
                                al(ND * (NS * eb * NF + padF())) + al(N * N + 6 * N) + al(NS * 2 * ND) +
                                al((int)((NFP + NS * 2 * ND) * 4 / sizeof(R)) + 1) + AL) +
           128;
  }
  static constexpr bool fits(int eb) { return NS * eb <= 1024 && smem_for(eb) <= kMaxSmem && eb * NF <= 256; }
  // FP64: largest power of two <= 32 with NS*EB <= 160, at least 2, times
  // 2^V (at most 32, halved until it fits).
  // FP32: 128/NS rounded down to a power of two, at least 4 (16-byte
  // offsets), times 2^V, at most 32, halved until it fits.
  static constexpr int eb64_base() {
    return NS * 32 <= 160 ? 32 : NS * 16 <= 160 ? 16 : NS * 8 <= 160 ? 8 : NS * 4 <= 160 ? 4 : 2;
  }
  static constexpr int eb64() { return (eb64_base() << V) > 32 ? 32 : (eb64_base() << V); }
  static constexpr int eb32_want() {
    return (pow2_floor(128 / NS) < 4 ? 4 : pow2_floor(128 / NS)) << V > 32
               ? 32
               : (pow2_floor(128 / NS) < 4 ? 4 : pow2_floor(128 / NS)) << V;
  }
  static constexpr int shrink(int eb) { return (eb <= 4 || fits(eb)) ? eb : shrink(eb / 2); }
  static constexpr int shrink64(int eb) { return (eb <= 2 || fits(eb)) ? eb : shrink64(eb / 2); }
  static constexpr int EB = F32 ? shrink(eb32_want()) : shrink64(eb64());
  static constexpr int NT = NS * EB;
  static constexpr int ROW = EB * NF;
  // the flux-point phases take one line (both of its ends) per thread where
  // one flux point per thread would need more than one round of the CTA
  static constexpr bool PAIR = NFP * EB > NT;
  // 3-D: the divergence and the extrapolated normal flux in one pass per
  // (line, element) over the line's flux values (LP), instead of a pass per
  // solution point for the divergence and one per line for the flux points
  // (3-D P3 32^3: FP32 element stage 0.1142 -> 0.1130 ms, FP64 0.1830 ->
  // 0.1818 ms with the register cap below; NS TGV 40^3 P4 1.047 -> 1.032 ms
  // FP64, 0.525 -> 0.509 ms FP32); FP64 inviscid at P2 and P3, where the
  // register cap below keeps the CTAs per SM with a few bytes spilled (at P0
  // and P1 the line pass would raise the registers from 72-80 to 96-126)
  static constexpr bool LP = ND == 3 && (F32 || VS || (P >= 2 && P <= 3));
  // the line pass also applies the correction from the line's two ends (the
  // solution points then need no pass over the flux-point records): FP32
  // (3-D P3 32^3 element stage 0.1113 -> 0.1026 ms; NS TGV 40^3 P4 0.500 ->
  // 0.476 ms); in FP64 the registers it needs cost more than it saves
  // (inviscid P3: 144 bytes spilled under the cap; viscous P4: 1.032 ->
  // 1.051 ms)
  static constexpr bool LPC = LP && F32;
  static constexpr int SLAB = NS * ROW + padF();  // one dimension's flux tile
  static constexpr int O_U = 0;
  static constexpr int O_U0 = O_U + al(NS * ROW);
  static constexpr int O_ACC = O_U0 + (LEAN ? 0 : al(NS * ROW));
  static constexpr int O_CMP = O_ACC + al(NS * ROW);
  static constexpr int O_FN = O_CMP + (F32 ? al(NS * ROW) : 0);
  static constexpr int O_DET = O_FN + al(NFP * ROW);
  static constexpr int O_J = O_DET + al(NS * EB);
  static constexpr int O_F = LEAN ? O_J : O_J + al(ND * NS * EB * ND);
  static constexpr int O_TAB = O_F + (al(ND * SLAB) > al(ND * NS * EB * ND) ? al(ND * SLAB) : al(ND * NS * EB * ND));
  // correction tables (corrVal [NS][2ND], corrFpt [NS][2ND]): inviscid
  // stages read them through L1 from global memory instead of staging them
  // (4.6 KB per FP64 CTA at 3-D P3, one more CTA per SM)
  static constexpr bool GTAB = !VS;
  static constexpr int NCT = GTAB ? 0 : NS * 2 * ND;
  static constexpr int O_CV = O_TAB + al(N * N + 6 * N);
  static constexpr int O_IDX = O_CV + al(NCT);  // ints: fpt line [NFP], corrFpt [NCT], line ends [NFP/2]
  static constexpr int O_BAR = O_IDX + al((int)((NFP + NCT + NFP / 2) * 4 / sizeof(R)) + 1);
  static constexpr size_t SMEM = sizeof(R) * (size_t)(O_BAR + AL) + 128;
  static_assert(SMEM <= kMaxSmem, "TMA tile set does not fit in shared memory");
  static_assert(NT <= 1024, "too many threads");
  // minimum CTAs per SM for the register allocation (0: none): the FP64
  // inviscid line pass holds a line's N records in registers, which uncapped
  // (100 registers at P3) costs a CTA per SM (0.205 ms instead of 0.182)
  static constexpr int CTAS = (int)((228 * 1024) / (SMEM + 1024));
  static constexpr int MINB = (LP && !F32 && !VS && 65536 / (NT * CTAS) >= 80) ? CTAS : 0;
  static_assert(!F32 || EB % 4 == 0, "FP32 tiles need 16-byte x offsets");
};

// s + e = a + b exactly (Knuth's TwoSum); the intrinsics keep the compiler
// from contracting or reassociating the steps.
__device__ __forceinline__ void two_sum(float a, float b, float &s, float &e) {
  s = __fadd_rn(a, b);
  const float bb = __fsub_rn(s, a);
  e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bb)), __fsub_rn(b, bb));
}

// One point's NF values of a tile row.  With 4 fields (2-D) the record is
// 16-byte aligned and moves as one 128-bit shared-memory access (two for
// FP64): four times fewer instructions than per-field accesses; otherwise
// per field.  A 128-bit access serves a quarter warp (8 lanes, normally 8
// consecutive records) per wavefront.  FP64 records are 32 bytes, so the
// first halves of 8 consecutive records fall on 16 of the 32 banks, twice
// each; every lane therefore takes its two halves in the order given by
// bit 7 of the record's address (bit 2 of its index), which pairs each
// first half with a second half of the record 128 bytes away and covers
// all 32 banks once (2-D FP64 element stage: 46 % of its shared-memory
// wavefronts were such conflicts).
template <int NF, typename R>
__device__ __forceinline__ int half_order(const R *p) {
  return (int)((reinterpret_cast<uintptr_t>(p) >> 7) & 1);
}
template <int NF, typename R>
__device__ __forceinline__ void ldp(const R *p, R (&v)[NF]) {
  if constexpr (NF == 4 && std::is_same<R, float>::value) {
    const float4 t = *reinterpret_cast<const float4 *>(p);
    v[0] = t.x, v[1] = t.y, v[2] = t.z, v[3] = t.w;
  } else if constexpr (NF == 4 && std::is_same<R, double>::value) {
    const int h = half_order<NF, R>(p);
    const double2 a = reinterpret_cast<const double2 *>(p)[h], b = reinterpret_cast<const double2 *>(p)[h ^ 1];
    v[0] = h ? b.x : a.x, v[1] = h ? b.y : a.y, v[2] = h ? a.x : b.x, v[3] = h ? a.y : b.y;
  } else {
#pragma unroll
    for (int k = 0; k < NF; k++) v[k] = p[k];
  }
}
// One row of a point's metric (ND values of JGinv); in 2-D the pair moves as
// one 8- or 16-byte access, which keeps consecutive lanes on consecutive
// banks (two scalar accesses at a 2-value stride conflict two ways).
template <int ND, typename R>
__device__ __forceinline__ void ldj(const R *p, R (&v)[ND]) {
  if constexpr (ND == 2 && std::is_same<R, double>::value) {
    const double2 t = *reinterpret_cast<const double2 *>(p);
    v[0] = t.x, v[1] = t.y;
  } else if constexpr (ND == 2 && std::is_same<R, float>::value) {
    const float2 t = *reinterpret_cast<const float2 *>(p);
    v[0] = t.x, v[1] = t.y;
  } else {
#pragma unroll
    for (int d = 0; d < ND; d++) v[d] = p[d];
  }
}
template <int NF, typename R>
__device__ __forceinline__ void stp(R *p, const R (&v)[NF]) {
  if constexpr (NF == 4 && std::is_same<R, float>::value) {
    *reinterpret_cast<float4 *>(p) = make_float4(v[0], v[1], v[2], v[3]);
  } else if constexpr (NF == 4 && std::is_same<R, double>::value) {
    const int h = half_order<NF, R>(p);
    reinterpret_cast<double2 *>(p)[h] = h ? make_double2(v[2], v[3]) : make_double2(v[0], v[1]);
    reinterpret_cast<double2 *>(p)[h ^ 1] = h ? make_double2(v[0], v[1]) : make_double2(v[2], v[3]);
  } else {
#pragma unroll
    for (int k = 0; k < NF; k++) p[k] = v[k];
  }
}

template <int ND, int P, typename R, int V, bool VISC>
__global__ void __launch_bounds__(Tm<ND, P, R, V, VISC>::NT, Tm<ND, P, R, V, VISC>::MINB) k_elem_tma(ElemArgsT<R> a, TpTablesT<R> t,
                                                                  const __grid_constant__ TmaMaps mp) {
  pdl_wait();
  pdl_trigger();
  using T = Tm<ND, P, R, V, VISC>;
  constexpr bool F32 = T::F32;
  constexpr bool LEAN = T::LEAN;
  constexpr int N = T::N, NF = T::NF, NS = T::NS, NFP = T::NFP, EB = T::EB, NT = T::NT, ROW = T::ROW;
  // viscous stages load the gradient into the flux tile as one dense box, so
  // they keep the flux tile unpadded; otherwise the new state is copied into
  // the padded flux tile for the extrapolation (E)
  constexpr bool PADDED = !VISC && T::PADDED;
  constexpr int SL = VISC ? NS * ROW : T::SLAB;
  // offset of point p of dimension d's flux tile
  const auto fidx = [](int d, int p) {
    if constexpr (PADDED)
      return d * SL + p * ROW + (p / N) * T::PADR + (p / (N * N)) * T::PADP;
    else
      return (d * NS + p) * ROW;
  };
  extern __shared__ __align__(128) unsigned char smem_bytes[];
  // tiles start on 128-byte boundaries relative to an aligned base
  R *smem = reinterpret_cast<R *>((reinterpret_cast<uintptr_t>(smem_bytes) + 127) & ~uintptr_t(127));
  R *sU = smem + T::O_U;
  R *sU0 = smem + T::O_U0;  // not in the lean tile set
  R *sAcc = smem + T::O_ACC;
  R *sCmp = smem + T::O_CMP;  // precision form only
  R *sFn = smem + T::O_FN;    // Fn -> Fn - extrapolated flux -> new U_fpts
  R *sJ = smem + T::O_J;      // [ND][NS][EB*ND]
  R *sDet = smem + T::O_DET;  // [NS][EB]
  R *sF = smem + T::O_F;      // [ND][SL]: point p of dimension d at fidx(d, p)
  R *sD = smem + T::O_TAB;
  R *sE = sD + N * N;
  R *sEF = sE + 2 * N;
  R *sCg = sEF + 2 * N;  // correction values by side and index along the line (LP)
  R *sCV = smem + T::O_CV;
  int *sLine = reinterpret_cast<int *>(smem + T::O_IDX);  // base | dn << 16 | side << 20
  int *sCF = sLine + NFP;
  int *sPair = sCF + T::NCT;  // side-0 fpt | side-1 fpt << 16 of each line
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem + T::O_BAR);

  const int E = a.E;
  const int e0 = blockIdx.x * EB;
  const int nValid = min(EB, E - e0);
  const int tid = threadIdx.x;
  const int s = tid / EB, el = tid - (tid / EB) * EB;
  const int e = e0 + el;
  const bool valid = el < nValid;

  // the last stage of the step: the precision form adds the increments to
  // the compensated state there
  const bool finalStage = a.mode == MODE_RK_FINAL || (a.mode == MODE_JAMESON && a.stage == a.nRK - 1);
  const bool needU0 = ((a.mode == MODE_RK_STAGE || a.mode == MODE_JAMESON) && a.stage > 0) ||
                      (F32 && a.mode == MODE_RK_FINAL && a.nRK > 1);
  const bool needAcc = (a.mode == MODE_RK_STAGE && a.stage > 0) || (a.mode == MODE_RK_FINAL && a.nRK > 1);
  const bool needCmp = F32 && finalStage;
  const bool needDet = a.mode != MODE_RESIDUAL;
  // the time step, loaded now so its latency hides behind the tile loads
  const double dtIn = a.mode == MODE_RESIDUAL ? 0.0 : (a.eleDt ? (valid ? a.eleDt[e] : 0.0) : *a.dt);

  // two transaction barriers: bar[0] for what the flux needs (U, JGinv),
  // bar[1] for what the correction and update need, so the second batch
  // lands while the flux and divergence are computed
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (tid == 0) {
    mbar_arrive_expect_tx(&bar[0], sizeof(R) * (NS * ROW + ND * NS * EB * ND + (VISC ? ND * NS * ROW : 0)));
    tma_load_2d(sU, &mp.U, e0 * NF, 0, &bar[0]);
    tma_load_3d(sJ, &mp.J, e0 * ND, 0, 0, &bar[0]);
    // viscous: the physical gradient lands in the flux tile, which the flux
    // phase then overwrites point by point
    if (VISC) tma_load_3d(sF, &mp.dUs, e0 * NF, 0, 0, &bar[0]);
    uint32_t bytes = sizeof(R) * NFP * ROW;
    if (needU0 && !LEAN) bytes += sizeof(R) * NS * ROW;
    if (needAcc) bytes += sizeof(R) * NS * ROW;
    if (needCmp) bytes += sizeof(R) * NS * ROW;
    if (needDet) bytes += sizeof(R) * NS * EB;
    mbar_arrive_expect_tx(&bar[1], bytes);
    tma_load_2d(sFn, &mp.Fn, e0 * NF, 0, &bar[1]);
    if (needU0 && !LEAN) tma_load_2d(sU0, &mp.U0, e0 * NF, 0, &bar[1]);
    if (needAcc) tma_load_2d(sAcc, &mp.acc, e0 * NF, 0, &bar[1]);
    if (needCmp) tma_load_2d(sCmp, &mp.comp, e0 * NF, 0, &bar[1]);
    if (needDet) tma_load_2d(sDet, &mp.det, e0, 0, &bar[1]);
  }
  for (int i = tid; i < N * N; i += NT) sD[i] = t.D[i];
  for (int i = tid; i < 2 * N; i += NT) {
    sE[i] = t.E1[i];
    sEF[i] = t.EFn1[i];
    if (T::LPC) sCg[i] = t.lineCorr[i];
  }
  for (int i = tid; i < NFP; i += NT) sLine[i] = t.fptBase[i] | (t.fptDn[i] << 16) | (t.fptSide[i] << 20);
  for (int i = tid; i < NFP / 2; i += NT) sPair[i] = t.linePair[i];
  if constexpr (!T::GTAB)
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
    R Fp[ND][NF];
    R u[NF];
    ldp<NF, R>(&sU[s * ROW + el * NF], u);
    if (valid) {
      inviscid_flux<ND, R>(u, Fp, R(a.gamma));
      if (VISC) {
        // physical viscous flux added to the physical inviscid flux
        // (reference: solver.cpp:777-811)
        R gU[ND][NF], Fv[ND][NF];
#pragma unroll
        for (int d = 0; d < ND; d++) ldp<NF, R>(&sF[(d * NS + s) * ROW + el * NF], gU[d]);
        viscous_flux<ND, R>(u, gU, a.ph, Fv);
#pragma unroll
        for (int d = 0; d < ND; d++)
#pragma unroll
          for (int k = 0; k < NF; k++) Fp[d][k] = Fv[d][k] + Fp[d][k];
      }
    } else {
#pragma unroll
      for (int d = 0; d < ND; d++)
#pragma unroll
        for (int k = 0; k < NF; k++) Fp[d][k] = R(0);
    }
    if constexpr (LEAN) {
      // every thread transforms its flux before any writes the flux tile,
      // which overlays the metric tile
      R Fr[ND][NF];
#pragma unroll
      for (int d1 = 0; d1 < ND; d1++) {
        R Jr[ND];
        ldj<ND, R>(&sJ[(d1 * NS + s) * EB * ND + el * ND], Jr);
#pragma unroll
        for (int k = 0; k < NF; k++) {
          R f = R(0);
#pragma unroll
          for (int d2 = 0; d2 < ND; d2++) f += Jr[d2] * Fp[d2][k];
          Fr[d1][k] = f;
          if (a.F_dbg && valid) a.F_dbg[(((long long)d1 * NS + s) * E + e) * NF + k] = f;
        }
      }
      __syncthreads();
#pragma unroll
      for (int d1 = 0; d1 < ND; d1++) stp<NF, R>(&sF[fidx(d1, s) + el * NF], Fr[d1]);
    } else {
#pragma unroll
      for (int d1 = 0; d1 < ND; d1++) {
        R Jr[ND];
        ldj<ND, R>(&sJ[(d1 * NS + s) * EB * ND + el * ND], Jr);
        R fk[NF];
#pragma unroll
        for (int k = 0; k < NF; k++) {
          R f = R(0);
#pragma unroll
          for (int d2 = 0; d2 < ND; d2++) f += Jr[d2] * Fp[d2][k];
          fk[k] = f;
          if (a.F_dbg && valid) a.F_dbg[(((long long)d1 * NS + s) * E + e) * NF + k] = f;
        }
        stp<NF, R>(&sF[fidx(d1, s) + el * NF], fk);
      }
    }
  }
  __syncthreads();

  // C1: flux divergence at (s, el) (LP: formed per line below)
  int idx3[3];
  idx3[0] = s % N;
  idx3[1] = ND > 1 ? (s / N) % N : 0;
  idx3[2] = ND > 2 ? s / (N * N) : 0;
  R div[NF];
#pragma unroll
  for (int d = 0; d < (T::LP ? 0 : ND); d++) {
    const int stride = d == 0 ? 1 : (d == 1 ? N : N * N);
    const int base = s - idx3[d] * stride;
    const R *Dr = &sD[idx3[d] * N];
    R acc[NF];
#pragma unroll
    for (int k = 0; k < NF; k++) acc[k] = R(0);
#pragma unroll
    for (int m = 0; m < N; m++) {
      const R dv = Dr[m];
      R x[NF];
      ldp<NF, R>(&sF[fidx(d, base + m * stride) + el * NF], x);
#pragma unroll
      for (int k = 0; k < NF; k++) acc[k] += dv * x[k];
    }
#pragma unroll
    for (int k = 0; k < NF; k++) div[k] = d == 0 ? acc[k] : div[k] + acc[k];
  }

  // lean tile set: this point's RK base state straight from global memory,
  // issued now so it lands while the extrapolated flux is formed
  R gU0[NF];
  if constexpr (LEAN) {
#pragma unroll
    for (int k = 0; k < NF; k++) gU0[k] = (needU0 && valid) ? a.U0[((long long)s * E + e) * NF + k] : R(0);
  }

  if (!mbar_wait_bounded(&bar[1], 0, 1u << 22)) {
    if (a.err) atomicOr(a.err, 1);
    mbar_wait_bounded(&bar[1], 0, 1u << 22);
    if (tid == 0) tma_wait_read_all();
    return;
  }

  constexpr int NE = T::PAIR ? 2 : 1;  // flux points per work item
  if constexpr (T::LPC) {
    // C (LP): per (line, element), the line's N flux values of its
    // direction once into registers; Fn - extrapolated normal flux at both
    // of its ends; then at its N points the divergence along the line plus
    // the correction from both ends, which replaces the flux values in the
    // flux tile (only this item reads them)
    for (int it = tid; it < (NFP / 2) * EB; it += NT) {
      const int l = it / EB, fe = it - (it / EB) * EB;
      const int pr = sPair[l];
      const int ln = sLine[pr & 0xffff];
      const int base = ln & 0xffff, dn = (ln >> 16) & 0xf;
      const int stride = dn == 0 ? 1 : (dn == 1 ? N : N * N);
      R x[N][NF];
#pragma unroll
      for (int m = 0; m < N; m++) ldp<NF, R>(&sF[fidx(dn, base + m * stride) + fe * NF], x[m]);
      R q[2][NF];
#pragma unroll
      for (int j = 0; j < 2; j++) {
        R acc[NF];
#pragma unroll
        for (int k = 0; k < NF; k++) acc[k] = R(0);
#pragma unroll
        for (int m = 0; m < N; m++) {
          const R ev = sEF[j * N + m];
#pragma unroll
          for (int k = 0; k < NF; k++) acc[k] += ev * x[m][k];
        }
        const int f = j ? pr >> 16 : pr & 0xffff;
        ldp<NF, R>(&sFn[f * ROW + fe * NF], q[j]);
#pragma unroll
        for (int k = 0; k < NF; k++) {
          q[j][k] = q[j][k] - acc[k];
          if (a.disFn_dbg && fe < nValid) a.disFn_dbg[((long long)f * E + e0 + fe) * NF + k] = q[j][k];
        }
      }
#pragma unroll
      for (int i = 0; i < N; i++) {
        R acc[NF];
#pragma unroll
        for (int k = 0; k < NF; k++) acc[k] = R(0);
#pragma unroll
        for (int m = 0; m < N; m++) {
          const R dv = sD[i * N + m];
#pragma unroll
          for (int k = 0; k < NF; k++) acc[k] += dv * x[m][k];
        }
        const R c0 = sCg[i], c1 = sCg[N + i];
#pragma unroll
        for (int k = 0; k < NF; k++) {
          R c = c0 * q[0][k];
          c += c1 * q[1][k];
          acc[k] = c + acc[k];
        }
        stp<NF, R>(&sF[fidx(dn, base + i * stride) + fe * NF], acc);
      }
    }
  }
  if constexpr (T::LP && !T::LPC) {
    // C (LP without the correction): the divergence along the line at its N
    // points replaces the flux values in the flux tile, and Fn - extrapolated
    // normal flux is formed in place at both ends for the correction in D
    for (int it = tid; it < (NFP / 2) * EB; it += NT) {
      const int l = it / EB, fe = it - (it / EB) * EB;
      const int pr = sPair[l];
      const int ln = sLine[pr & 0xffff];
      const int base = ln & 0xffff, dn = (ln >> 16) & 0xf;
      const int stride = dn == 0 ? 1 : (dn == 1 ? N : N * N);
      R x[N][NF];
#pragma unroll
      for (int m = 0; m < N; m++) ldp<NF, R>(&sF[fidx(dn, base + m * stride) + fe * NF], x[m]);
#pragma unroll
      for (int i = 0; i < N; i++) {
        R acc[NF];
#pragma unroll
        for (int k = 0; k < NF; k++) acc[k] = R(0);
#pragma unroll
        for (int m = 0; m < N; m++) {
          const R dv = sD[i * N + m];
#pragma unroll
          for (int k = 0; k < NF; k++) acc[k] += dv * x[m][k];
        }
        stp<NF, R>(&sF[fidx(dn, base + i * stride) + fe * NF], acc);
      }
#pragma unroll
      for (int j = 0; j < 2; j++) {
        R acc[NF];
#pragma unroll
        for (int k = 0; k < NF; k++) acc[k] = R(0);
#pragma unroll
        for (int m = 0; m < N; m++) {
          const R ev = sEF[j * N + m];
#pragma unroll
          for (int k = 0; k < NF; k++) acc[k] += ev * x[m][k];
        }
        const int f = j ? pr >> 16 : pr & 0xffff;
        R *q = &sFn[f * ROW + fe * NF];
        R qv[NF];
        ldp<NF, R>(q, qv);
#pragma unroll
        for (int k = 0; k < NF; k++) {
          qv[k] = qv[k] - acc[k];
          if (a.disFn_dbg && fe < nValid) a.disFn_dbg[((long long)f * E + e0 + fe) * NF + k] = qv[k];
        }
        stp<NF, R>(q, qv);
      }
    }
  }
  // C2: Fn - extrapolated normal flux, in place in the Fn tile, per flux
  // point or (PAIR) per line: one pass over a line's points gives both ends
  for (int it = tid; !T::LP && it < (NFP / NE) * EB; it += NT) {
    const int l = it / EB, fe = it - (it / EB) * EB;
    const int pr = T::PAIR ? sPair[l] : l;  // side-0 fpt | side-1 fpt << 16, or the fpt
    const int ln = sLine[pr & 0xffff];
    const int base = ln & 0xffff, dn = (ln >> 16) & 0xf, side0 = T::PAIR ? 0 : ln >> 20;
    const int stride = dn == 0 ? 1 : (dn == 1 ? N : N * N);
    R acc[NE][NF];
#pragma unroll
    for (int j = 0; j < NE; j++)
#pragma unroll
      for (int k = 0; k < NF; k++) acc[j][k] = R(0);
#pragma unroll
    for (int m = 0; m < N; m++) {
      R x[NF];
      ldp<NF, R>(&sF[fidx(dn, base + m * stride) + fe * NF], x);
#pragma unroll
      for (int j = 0; j < NE; j++) {
        const R ev = sEF[(j ? 1 : side0) * N + m];
#pragma unroll
        for (int k = 0; k < NF; k++) acc[j][k] += ev * x[k];
      }
    }
#pragma unroll
    for (int j = 0; j < NE; j++) {
      const int f = j ? pr >> 16 : pr & 0xffff;
      R *q = &sFn[f * ROW + fe * NF];
      R qv[NF];
      ldp<NF, R>(q, qv);
#pragma unroll
      for (int k = 0; k < NF; k++) {
        qv[k] = qv[k] - acc[j][k];
        if (a.disFn_dbg && fe < nValid) a.disFn_dbg[((long long)f * E + e0 + fe) * NF + k] = qv[k];
      }
      stp<NF, R>(q, qv);
    }
  }
  if (tid == 0) tma_wait_read_all();  // the U0 store has read sU
  __syncthreads();
  if constexpr (T::LP) {
    // the divergence at (s, el): the three directions' parts, x, y, z
#pragma unroll
    for (int d = 0; d < ND; d++) {
      R x[NF];
      ldp<NF, R>(&sF[fidx(d, s) + el * NF], x);
#pragma unroll
      for (int k = 0; k < NF; k++) div[k] = d == 0 ? x[k] : div[k] + x[k];
    }
  }

  // D: correction (LPC: already in the line sums) and RK update at (s, el),
  // in place in sU / sAcc / sCmp
  {
    R cq[NF];
#pragma unroll
    for (int k = 0; k < NF; k++) cq[k] = R(0);
#pragma unroll
    for (int fc = 0; fc < (T::LPC ? 0 : 2 * ND); fc++) {
      const int fp = T::GTAB ? __ldg(&t.corrFpt[s * 2 * ND + fc]) : sCF[s * 2 * ND + fc];
      const R cv = T::GTAB ? __ldg(&t.corrVal[s * 2 * ND + fc]) : sCV[s * 2 * ND + fc];
      R x[NF];
      ldp<NF, R>(&sFn[fp * ROW + el * NF], x);
#pragma unroll
      for (int k = 0; k < NF; k++) cq[k] += cv * x[k];
    }
    // one reciprocal per point instead of a division per update term
    const R rdJ = needDet ? R(1.0) / sDet[s * EB + el] : R(1.0);
    const R dt = R(dtIn);
    const R rka = R(a.rka_next), rkb = R(a.rkb);
    const int l0 = s * ROW + el * NF;
    R vU[NF], vU0[NF], vAcc[NF], vCmp[NF];
    if (a.mode != MODE_RESIDUAL) {
      ldp<NF, R>(&sU[l0], vU);
      if (needU0) {
        if constexpr (LEAN) {
#pragma unroll
          for (int k = 0; k < NF; k++) vU0[k] = gU0[k];
        } else {
          ldp<NF, R>(&sU0[l0], vU0);
        }
      }
      if (needAcc) ldp<NF, R>(&sAcc[l0], vAcc);
      if (needCmp) ldp<NF, R>(&sCmp[l0], vCmp);
    }
#pragma unroll
    for (int k = 0; k < NF; k++) {
      const long long gi = ((long long)s * E + e) * NF + k;
      R dv = cq[k] + div[k];
      if (a.divF_out && valid) a.divF_out[gi] = dv;
      if (a.mode == MODE_RESIDUAL) continue;
      if (a.src && valid) dv = dv + a.src[gi];
      const R u = vU[k];
      R unew;
      if constexpr (!F32) {
        if (a.mode == MODE_RK_STAGE) {
          const R u0 = a.stage == 0 ? u : vU0[k];
          unew = u0 - rka * dv * rdJ * dt;
          const R base = a.stage == 0 ? u0 : vAcc[k];
          vAcc[k] = base - rkb * dv * rdJ * dt;
        } else if (a.mode == MODE_RK_FINAL) {
          const R base = a.nRK == 1 ? u : vAcc[k];
          unew = base - rkb * dv * rdJ * dt;
        } else {
          const R u0 = a.stage == 0 ? u : vU0[k];
          unew = u0 - rka * dv * rdJ * dt;
        }
      } else {
        const R inc = dv * rdJ * dt;
        if (a.mode == MODE_RK_STAGE) {
          const R u0 = a.stage == 0 ? u : vU0[k];
          unew = u0 - rka * inc;
          vAcc[k] = (a.stage == 0 ? R(0) : vAcc[k]) - rkb * inc;
        } else if (finalStage) {
          const R u0 = (a.mode == MODE_RK_FINAL && a.nRK > 1) || (a.mode == MODE_JAMESON && a.stage > 0) ? vU0[k] : u;
          const R sum = a.mode == MODE_RK_FINAL ? (a.nRK > 1 ? vAcc[k] : R(0)) - rkb * inc : -(rka * inc);
          R c;
          two_sum(u0, vCmp[k] + sum, unew, c);
          vCmp[k] = c;
        } else {
          const R u0 = a.stage == 0 ? u : vU0[k];
          unew = u0 - rka * inc;
        }
      }
      vU[k] = unew;
    }
    if (a.mode != MODE_RESIDUAL) {
      stp<NF, R>(&sU[l0], vU);
      if (PADDED) stp<NF, R>(&sF[fidx(0, s) + el * NF], vU);  // the flux tile is dead after C2
      if (a.mode == MODE_RK_STAGE) stp<NF, R>(&sAcc[l0], vAcc);
      if (needCmp) stp<NF, R>(&sCmp[l0], vCmp);
    }
  }
  if (a.mode == MODE_RESIDUAL) return;
  fence_async_smem();
  __syncthreads();
  if (tid == 0) {
    tma_store_2d(&mp.U, e0 * NF, 0, sU);
    if (a.mode == MODE_RK_STAGE) tma_store_2d(&mp.acc, e0 * NF, 0, sAcc);
    if (needCmp) tma_store_2d(&mp.comp, e0 * NF, 0, sCmp);
    tma_commit();
  }
  if (!a.Ufpts_out) {
    if (tid == 0) tma_wait_read_all();
    return;
  }

  // E: new state at the flux points, into the Fn tile (per flux point or,
  // PAIR, per line as in C2)
  for (int it = tid; it < (NFP / NE) * EB; it += NT) {
    const int l = it / EB, fe = it - (it / EB) * EB;
    const int pr = T::PAIR ? sPair[l] : l;
    const int ln = sLine[pr & 0xffff];
    const int base = ln & 0xffff, dn = (ln >> 16) & 0xf, side0 = T::PAIR ? 0 : ln >> 20;
    const int stride = dn == 0 ? 1 : (dn == 1 ? N : N * N);
    R acc[NE][NF];
#pragma unroll
    for (int j = 0; j < NE; j++)
#pragma unroll
      for (int k = 0; k < NF; k++) acc[j][k] = R(0);
#pragma unroll
    for (int m = 0; m < N; m++) {
      R x[NF];
      if (PADDED)
        ldp<NF, R>(&sF[fidx(0, base + m * stride) + fe * NF], x);
      else
        ldp<NF, R>(&sU[(base + m * stride) * ROW + fe * NF], x);
#pragma unroll
      for (int j = 0; j < NE; j++) {
        const R ev = sE[(j ? 1 : side0) * N + m];
#pragma unroll
        for (int k = 0; k < NF; k++) acc[j][k] += ev * x[k];
      }
    }
#pragma unroll
    for (int j = 0; j < NE; j++) stp<NF, R>(&sFn[(j ? pr >> 16 : pr & 0xffff) * ROW + fe * NF], acc[j]);
  }
  fence_async_smem();
  __syncthreads();
  if (tid == 0) {
    tma_store_2d(&mp.Ufpts, e0 * NF, 0, sFn);
    tma_commit();
    tma_wait_read_all();
  }
}

template <int ND, int P, typename R, int V, bool VISC = false>
void launch_tma(const ElemArgsT<R> &a, const TpTablesT<R> &t, const TmaMaps &m, cudaStream_t st) {
  using T = Tm<ND, P, R, V, VISC>;
  static std::atomic<unsigned long long> attrDev{0};
  smem_attr(k_elem_tma<ND, P, R, V, VISC>, (int)T::SMEM, attrDev);
  int g = (a.E + T::EB - 1) / T::EB;
  launch_k(k_elem_tma<ND, P, R, V, VISC>, g, T::NT, T::SMEM, st, a, t, m);
}

// The CTAs per SM the tile layouts are built for at 3-D P3 (228 KB of shared
// memory per SM, 1 KB of it reserved per CTA): the lean FP64 set, six
// 2-element or three 4-element CTAs; FP32 4-element tiles, four.
constexpr bool ctas_fit(size_t smem, int ctas) { return (smem + 1024) * ctas <= 228 * 1024; }
static_assert(ctas_fit(Tm<3, 3, double, 0>::SMEM, 6) && Tm<3, 3, double, 0>::EB == 2, "FP64 P3 2-element tiles");
static_assert(ctas_fit(Tm<3, 3, double, 1>::SMEM, 3) && Tm<3, 3, double, 1>::EB == 4, "FP64 P3 4-element tiles");
static_assert(ctas_fit(Tm<3, 3, float, 0>::SMEM, 4) && Tm<3, 3, float, 0>::EB == 4, "FP32 P3 4-element tiles");

// (nDims, order) -> compile-time case; variants only for the precision form
#define FR_TM_ORDERS(X) X(2, 0) X(2, 1) X(2, 2) X(2, 3) X(2, 4) X(2, 5) X(3, 0) X(3, 1) X(3, 2) X(3, 3) X(3, 4) X(3, 5)

template <typename R, int V>
int eb_of(int nDims, int order) {
#define FR_TM_EB(ND, P) \
  if (nDims == ND && order == P) return Tm<ND, P, R, V>::EB;
  FR_TM_ORDERS(FR_TM_EB)
#undef FR_TM_EB
  return 0;
}
template <typename R, int V>
size_t smem_of(int nDims, int order) {
#define FR_TM_SM(ND, P) \
  if (nDims == ND && order == P) return Tm<ND, P, R, V>::SMEM;
  FR_TM_ORDERS(FR_TM_SM)
#undef FR_TM_SM
  return 0;
}
template <typename R, int V>
void launch_v(int nDims, int order, const ElemArgsT<R> &a, const TpTablesT<R> &t, const TmaMaps &m,
              cudaStream_t st) {
#define FR_TM_CASE(ND, P) \
  if (nDims == ND && order == P) return launch_tma<ND, P, R, V>(a, t, m, st);
  FR_TM_ORDERS(FR_TM_CASE)
#undef FR_TM_CASE
}


// Corrected, physical solution gradient at the solution points and its
// extrapolation to the flux points (reference: solver.cpp:1060-1158), one
// thread per (solution point, element) of a block of EB elements, all tiles
// moved by TMA: U, the LDG jumps dUc, JGinv and detJ in; dU_spts and dU_fpts
// out.  Same sums, in the same order, as k_elem_grad.
template <int ND, int P, typename R>
struct Tg2 {
  using T = Tm<ND, P, R, 0>;
  static constexpr int N = T::N, NF = T::NF, NS = T::NS, NFP = T::NFP, EB = T::EB, NT = T::NT, ROW = T::ROW;
  static constexpr bool PAIR = T::PAIR;
  static constexpr int AL = T::AL;
  static constexpr int al(int n) { return (n + AL - 1) / AL * AL; }
  // the flux-point gradient tile reuses the input tiles (U, dUc, JGinv,
  // detJ), dead once the gradient at the solution points is formed
  static constexpr int O_U = 0;
  static constexpr int O_C = O_U + al(NS * ROW);
  static constexpr int O_J = O_C + al(NFP * ROW);
  static constexpr int O_DET = O_J + al(ND * NS * EB * ND);
  static constexpr int IN_END = O_DET + al(NS * EB);
  static constexpr int O_GF = O_U;
  static constexpr int O_G = IN_END > al(ND * NFP * ROW) ? IN_END : al(ND * NFP * ROW);
  // 3-D: the reference gradient is formed per (line, element) with the
  // correction values by side and index along the line (GLP), so the
  // per-point correction tables are not staged
  static constexpr bool GLP = ND == 3;
  static constexpr int NCT = GLP ? 0 : NS * 2 * ND;
  static constexpr int O_TAB = O_G + al(ND * NS * ROW);
  static constexpr int O_CV = O_TAB + al(N * N + 4 * N);
  static constexpr int O_IDX = O_CV + al(NCT);
  static constexpr int O_BAR = O_IDX + al((int)((NFP + NCT + NFP / 2) * 4 / sizeof(R)) + 1);
  static constexpr size_t SMEM = sizeof(R) * (size_t)(O_BAR + AL) + 128;
  static_assert(SMEM <= kMaxSmem, "gradient tile set does not fit in shared memory");
};

template <int ND, int P, typename R>
__global__ void __launch_bounds__(Tg2<ND, P, R>::NT) k_grad_tma(int E, TpTablesT<R> t, unsigned int *err,
                                                                const __grid_constant__ TmaMaps mp) {
  pdl_wait();
  pdl_trigger();
  using T = Tg2<ND, P, R>;
  constexpr int N = T::N, NF = T::NF, NS = T::NS, NFP = T::NFP, EB = T::EB, NT = T::NT, ROW = T::ROW;
  extern __shared__ __align__(128) unsigned char smem_bytes[];
  R *smem = reinterpret_cast<R *>((reinterpret_cast<uintptr_t>(smem_bytes) + 127) & ~uintptr_t(127));
  R *sU = smem + T::O_U;
  R *sC = smem + T::O_C;      // [NFP][ROW] LDG jumps
  R *sJ = smem + T::O_J;      // [ND][NS][EB*ND]
  R *sDet = smem + T::O_DET;  // [NS][EB]
  R *sG = smem + T::O_G;      // [ND][NS][ROW] physical gradient
  R *sGf = smem + T::O_GF;    // [ND][NFP][ROW] at the flux points
  R *sD = smem + T::O_TAB;
  R *sE = sD + N * N;
  R *sCg = sE + 2 * N;  // GLP: correction values by side and index along the line
  R *sCV = smem + T::O_CV;
  int *sLine = reinterpret_cast<int *>(smem + T::O_IDX);
  int *sCF = sLine + NFP;
  int *sPair = sCF + T::NCT;  // side-0 fpt | side-1 fpt << 16 of each line
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem + T::O_BAR);

  const int e0 = blockIdx.x * EB;
  const int nValid = min(EB, E - e0);
  const int tid = threadIdx.x;
  const int s = tid / EB, el = tid - (tid / EB) * EB;
  const bool valid = el < nValid;

  if (tid == 0) {
    mbar_init(&bar[0], 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (tid == 0) {
    mbar_arrive_expect_tx(&bar[0], sizeof(R) * (NS * ROW + NFP * ROW + ND * NS * EB * ND + NS * EB));
    tma_load_2d(sU, &mp.U, e0 * NF, 0, &bar[0]);
    tma_load_2d(sC, &mp.dUc, e0 * NF, 0, &bar[0]);
    tma_load_3d(sJ, &mp.J, e0 * ND, 0, 0, &bar[0]);
    tma_load_2d(sDet, &mp.det, e0, 0, &bar[0]);
  }
  for (int i = tid; i < N * N; i += NT) sD[i] = t.D[i];
  for (int i = tid; i < 2 * N; i += NT) {
    sE[i] = t.E1[i];
    if (T::GLP) sCg[i] = t.lineCorr[i];
  }
  for (int i = tid; i < NFP; i += NT) sLine[i] = t.fptBase[i] | (t.fptDn[i] << 16) | (t.fptSide[i] << 20);
  for (int i = tid; i < NFP / 2; i += NT) sPair[i] = t.linePair[i];
  for (int i = tid; i < T::NCT; i += NT) {
    sCF[i] = t.corrFpt[i];
    sCV[i] = t.corrVal[i];
  }
  const bool ok = __syncthreads_and(mbar_wait_bounded(&bar[0], 0, 1u << 22));
  if (!ok) {
    if (tid == 0 && err) atomicOr(err, 1);
    mbar_wait_bounded(&bar[0], 0, 1u << 22);
    return;
  }

  R J[ND][ND];
#pragma unroll
  for (int d1 = 0; d1 < ND; d1++)
#pragma unroll
    for (int d2 = 0; d2 < ND; d2++) J[d1][d2] = valid ? sJ[(d1 * NS + s) * EB * ND + el * ND + d2] : R(0.0);
  const R invDet = valid ? R(1.) / sDet[s * EB + el] : R(0.0);
  int idx3[3];
  idx3[0] = s % N;
  idx3[1] = ND > 1 ? (s / N) % N : 0;
  idx3[2] = ND > 2 ? s / (N * N) : 0;
  R gr[ND][NF];
  if constexpr (T::GLP) {
    // per (line, element): the line's N states once into registers; at its N
    // points the reference gradient along the line plus the correction from
    // the jumps at its two ends, in the order of the per-point form (the two
    // faces normal to the line, the side-0 face first as in the hex face
    // numbering; corrVal times -1 on side 0), into sG[dn][point]
    for (int it = tid; it < (NFP / 2) * EB; it += NT) {
      const int l = it / EB, fe = it - (it / EB) * EB;
      const int pr = sPair[l];
      const int f0 = pr & 0xffff, f1 = pr >> 16;
      const int ln = sLine[f0];
      const int base = ln & 0xffff, dn = (ln >> 16) & 0xf;
      const int stride = dn == 0 ? 1 : (dn == 1 ? N : N * N);
      R x[N][NF], q0[NF], q1[NF];
#pragma unroll
      for (int m = 0; m < N; m++)
#pragma unroll
        for (int k = 0; k < NF; k++) x[m][k] = sU[(base + m * stride) * ROW + fe * NF + k];
#pragma unroll
      for (int k = 0; k < NF; k++) {
        q0[k] = sC[f0 * ROW + fe * NF + k];
        q1[k] = sC[f1 * ROW + fe * NF + k];
      }
#pragma unroll
      for (int i = 0; i < N; i++) {
        R acc[NF];
#pragma unroll
        for (int k = 0; k < NF; k++) acc[k] = R(0.0);
#pragma unroll
        for (int m = 0; m < N; m++) {
          const R dv = sD[i * N + m];
#pragma unroll
          for (int k = 0; k < NF; k++) acc[k] += dv * x[m][k];
        }
        const R cv0 = sCg[i] * -R(1.0), cv1 = sCg[N + i] * R(1.0);
#pragma unroll
        for (int k = 0; k < NF; k++) {
          R cq = R(0.0);
          cq += cv0 * q0[k];
          cq += cv1 * q1[k];
          sG[(dn * NS + base + i * stride) * ROW + fe * NF + k] = cq + acc[k];
        }
      }
    }
    __syncthreads();
#pragma unroll
    for (int d = 0; d < ND; d++)
#pragma unroll
      for (int k = 0; k < NF; k++) gr[d][k] = sG[(d * NS + s) * ROW + el * NF + k];
  }
#pragma unroll
  for (int d = 0; d < (T::GLP ? 0 : ND); d++) {
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
      const int fp = sCF[s * 2 * ND + fc];
      const int ln = sLine[fp];
      if (((ln >> 16) & 0xf) != d) continue;
      const R cv = sCV[s * 2 * ND + fc] * ((ln >> 20) ? R(1.0) : -R(1.0));
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
    }
  fence_async_smem();
  __syncthreads();  // the input tiles are dead from here on (sGf reuses them)
  if (tid == 0) {
    tma_store_3d(&mp.dUs, e0 * NF, 0, 0, sG);
    tma_commit();
  }
  // per flux point, or (PAIR) per line: both ends from one pass over it
  constexpr int NE = T::PAIR ? 2 : 1;
  for (int it = tid; it < (NFP / NE) * EB; it += NT) {
    const int l = it / EB, fe = it - (it / EB) * EB;
    const int pr = T::PAIR ? sPair[l] : l;
    const int ln = sLine[pr & 0xffff];
    const int base = ln & 0xffff, dn = (ln >> 16) & 0xf, side0 = T::PAIR ? 0 : ln >> 20;
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
        const int f = j ? pr >> 16 : pr & 0xffff;
#pragma unroll
        for (int k = 0; k < NF; k++) sGf[(d * NFP + f) * ROW + fe * NF + k] = acc[j][k];
      }
    }
  }
  fence_async_smem();
  __syncthreads();
  if (tid == 0) {
    tma_store_3d(&mp.dUf, e0 * NF, 0, 0, sGf);
    tma_commit();
    tma_wait_read_all();
  }
}

template <int ND, int P, typename R>
void launch_grad(int E, const TpTablesT<R> &t, const TmaMaps &m, unsigned int *err, cudaStream_t st) {
  using T = Tg2<ND, P, R>;
  static std::atomic<unsigned long long> attrDev{0};
  smem_attr(k_grad_tma<ND, P, R>, (int)T::SMEM, attrDev);
  launch_k(k_grad_tma<ND, P, R>, (E + T::EB - 1) / T::EB, T::NT, T::SMEM, st, E, t, err, m);
}

template <typename R>
void launch_v_visc(int nDims, int order, const ElemArgsT<R> &a, const TpTablesT<R> &t, const TmaMaps &m,
                   cudaStream_t st) {
#define FR_TMV_CASE(ND, P) \
  if (nDims == ND && order == P) return launch_tma<ND, P, R, 0, true>(a, t, m, st);
  FR_TM_ORDERS(FR_TMV_CASE)
#undef FR_TMV_CASE
}

}  // namespace

template <typename R>
void launch_element_stage_tma_visc(int nDims, int order, const ElemArgsT<R> &a, const TpTablesT<R> &t,
                                   const TmaMaps &m, cudaStream_t st) {
  if (a.E <= 0) return;
  launch_v_visc<R>(nDims, order, a, t, m, st);
}
template void launch_element_stage_tma_visc<double>(int, int, const ElemArgsT<double> &, const TpTablesT<double> &,
                                                    const TmaMaps &, cudaStream_t);
template void launch_element_stage_tma_visc<float>(int, int, const ElemArgsT<float> &, const TpTablesT<float> &,
                                                   const TmaMaps &, cudaStream_t);

template <typename R>
void launch_elem_grad_tma(int nDims, int order, int E, const TpTablesT<R> &t, const TmaMaps &m, unsigned int *err,
                          cudaStream_t st) {
  if (E <= 0) return;
#define FR_TG_CASE(ND, P) \
  if (nDims == ND && order == P) return launch_grad<ND, P, R>(E, t, m, err, st);
  FR_TM_ORDERS(FR_TG_CASE)
#undef FR_TG_CASE
}
template void launch_elem_grad_tma<double>(int, int, int, const TpTablesT<double> &, const TmaMaps &, unsigned int *,
                                           cudaStream_t);
template void launch_elem_grad_tma<float>(int, int, int, const TpTablesT<float> &, const TmaMaps &, unsigned int *,
                                          cudaStream_t);

int tma_variants(bool fp32) { return fp32 ? kFp32Variants : kFp64Variants; }

template <>
int tma_elems_per_block<double>(int nDims, int order, int v) {
  return v == 0 ? eb_of<double, 0>(nDims, order) : eb_of<double, 1>(nDims, order);
}
template <>
int tma_elems_per_block<float>(int nDims, int order, int v) {
  if (v == kFp32Variants) return tc_elems_per_block(nDims, order);  // the tensor-core variant
  return v == 0 ? eb_of<float, 0>(nDims, order) : v == 1 ? eb_of<float, 1>(nDims, order) : eb_of<float, 2>(nDims, order);
}
template <>
size_t tma_smem_bytes<double>(int nDims, int order, int v) {
  return v == 0 ? smem_of<double, 0>(nDims, order) : smem_of<double, 1>(nDims, order);
}
template <>
size_t tma_smem_bytes<float>(int nDims, int order, int v) {
  return v == 0 ? smem_of<float, 0>(nDims, order) : v == 1 ? smem_of<float, 1>(nDims, order) : smem_of<float, 2>(nDims, order);
}

template <>
void launch_element_stage_tma<double>(int nDims, int order, const ElemArgsT<double> &a, const TpTablesT<double> &t,
                                      const TmaMaps &m, cudaStream_t st, int v) {
  if (a.E <= 0) return;
  if (v == 0)
    launch_v<double, 0>(nDims, order, a, t, m, st);
  else
    launch_v<double, 1>(nDims, order, a, t, m, st);
}
template <>
void launch_element_stage_tma<float>(int nDims, int order, const ElemArgsT<float> &a, const TpTablesT<float> &t,
                                     const TmaMaps &m, cudaStream_t st, int v) {
  if (a.E <= 0) return;
  if (v == 0)
    launch_v<float, 0>(nDims, order, a, t, m, st);
  else if (v == 1)
    launch_v<float, 1>(nDims, order, a, t, m, st);
  else
    launch_v<float, 2>(nDims, order, a, t, m, st);
}

}  // namespace frk
