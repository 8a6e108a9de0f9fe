// Tensor-product element kernel (quads and hexes, orders 0..5), FP64 plain
// form and FP32 precision form.
//
// Same stage as k_element_stage (flux at the solution points, divergence,
// extrapolated normal flux, correction, RK update, extrapolation of the new
// state to the flux points; reference: solver.cpp:470-572, 707-736,
// 906-1058), with compile-time sizes: one thread per (solution point,
// element), all fields in registers, the 1-D operator tables in shared
// memory.  Every sum is the one the dense operator would form, over its
// nonzero terms in ascending column order.
#include <algorithm>
#include <atomic>
#include <type_traits>

#include "launch.cuh"
#include "stage.hpp"

namespace frk {

namespace {

constexpr int ipow(int b, int e) { return e == 0 ? 1 : b * ipow(b, e - 1); }

template <int ND, int P, typename R = double>
struct Tp {
  static constexpr int N = P + 1;
  static constexpr int NF = ND + 2;
  static constexpr int NS = ipow(N, ND);
  static constexpr int NPF = ipow(N, ND - 1);
  static constexpr int NFP = 2 * ND * NPF;
  static constexpr int EB = NS >= 256 ? 1 : (NS * 2 > 256 ? 1 : (NS * 4 > 256 ? 2 : (NS * 8 > 256 ? 4 : (NS * 16 > 256 ? 8 : (NS * 32 > 256 ? 16 : 32)))));
  static constexpr int NT = NS * EB;
  static constexpr int ROW = EB * NF;  // values per point row of a tile
  // flux-point phases per line (both ends) where one flux point per thread
  // would need more than one round of the block
  static constexpr bool PAIR = NFP * EB > NT;
  static constexpr size_t SMEM = sizeof(R) * ((size_t)ROW * (NS * (1 + ND) + NFP) + N * N + 4 * N);
};

// s + e = a + b exactly (TwoSum), not contracted or reassociated
__device__ __forceinline__ void two_sum_tp(float a, float b, float &s, float &e) {
  s = __fadd_rn(a, b);
  const float bb = __fsub_rn(s, a);
  e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bb)), __fsub_rn(b, bb));
}

// One element block (EB elements from element blk * EB) of the stage; the
// block's threads are threads 0..NT-1 of the CTA, and further threads of a
// larger CTA (the many-order kernel below) only take part in its barriers.
// LINES allows the per-line flux-point phases (the many-order kernel keeps
// one flux point per thread: its CTA holds every order's code, and the line
// form's registers for the small orders cost it a CTA per SM).
template <int ND, int P, bool VISC, typename R, bool LINES = true>
__device__ __forceinline__ void elem_tp_block(const ElemArgsT<R> &a, const TpTablesT<R> &t, int blk,
                                              unsigned char *smem_bytes) {
  using T = Tp<ND, P, R>;
  constexpr bool PAIR = LINES && T::PAIR;
  constexpr bool F32 = std::is_same<R, float>::value;
  constexpr int N = T::N, NF = T::NF, NS = T::NS, NFP = T::NFP, EB = T::EB, NT = T::NT, ROW = T::ROW;
  R *smem = reinterpret_cast<R *>(smem_bytes);
  R *sU = smem;                 // [NS][EB][NF]
  R *sF = sU + NS * ROW;        // [ND][NS][EB][NF]
  R *sQ = sF + ND * NS * ROW;   // [NFP][EB][NF]
  R *sD = sQ + NFP * ROW;       // [N][N]
  R *sE = sD + N * N;           // [2][N]
  R *sEF = sE + 2 * N;          // [2][N]

  const int E = a.E;
  const int e0 = blk * EB;
  const int nValid = min(EB, E - e0);
  const int tid = threadIdx.x;
  const bool act = tid < NT;  // a thread of this block's NT
  const int s = act ? tid / EB : 0, el = act ? tid - (tid / EB) * EB : 0;
  const int e = e0 + el;
  const bool valid = act && el < nValid;
  // the time step, loaded early so its latency overlaps the tile loads
  const double dtIn = a.eleDt ? (valid ? a.eleDt[e] : 0.0) : (a.mode != MODE_RESIDUAL ? *a.dt : 0.0);

  if (act) {
    for (int i = tid; i < N * N; i += NT) sD[i] = t.D[i];
    for (int i = tid; i < 2 * N; i += NT) {
      sE[i] = t.E1[i];
      sEF[i] = t.EFn1[i];
    }
    // A: state tile, coalesced along (element, field)
    for (int idx = tid; idx < NS * ROW; idx += NT) {
      const int ss = idx / ROW, r = idx - ss * ROW;
      sU[idx] = (r < nValid * NF) ? a.U[((long long)ss * E + e0) * NF + r] : R(1.0);
    }
  }
  R J[ND][ND];
#pragma unroll
  for (int d1 = 0; d1 < ND; d1++)
#pragma unroll
    for (int d2 = 0; d2 < ND; d2++)
      J[d1][d2] = valid ? a.JGinv[(((long long)d1 * NS + s) * E + e) * ND + d2] : R(0.0);
  __syncthreads();

  // B: reference-space flux at (s, el)
  if (act) {
    R Fp[ND][NF];
    const R *u = &sU[s * ROW + el * NF];
    if (valid) {
      inviscid_flux<ND, R>(u, Fp, R(a.gamma));
      if (VISC) {
        // physical viscous flux added to the physical inviscid flux
        // (reference: solver.cpp:777-811)
        R gU[ND][NF], Fv[ND][NF];
#pragma unroll
        for (int d = 0; d < ND; d++)
#pragma unroll
          for (int k = 0; k < NF; k++) gU[d][k] = a.dUs[d * a.dUsStride + ((long long)s * E + e) * NF + k];
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
        for (int k = 0; k < NF; k++) Fp[d][k] = R(0.0);
    }
#pragma unroll
    for (int d1 = 0; d1 < ND; d1++)
#pragma unroll
      for (int k = 0; k < NF; k++) {
        R f = R(0.0);
#pragma unroll
        for (int d2 = 0; d2 < ND; d2++) f += J[d1][d2] * Fp[d2][k];
        sF[(d1 * NS + s) * ROW + el * NF + k] = f;
        if (a.F_dbg && valid) a.F_dbg[(((long long)d1 * NS + s) * E + e) * NF + k] = f;
      }
  }
  __syncthreads();

  // C1: divergence at (s, el): sum over d of D-lines (threads past NT read
  // the first point's lines and use nothing)
  int idx3[3];
  idx3[0] = s % N;
  idx3[1] = ND > 1 ? (s / N) % N : 0;
  idx3[2] = ND > 2 ? s / (N * N) : 0;
  R div[NF];
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
      const R *x = &sF[(d * NS + base + m * stride) * ROW + el * NF];
#pragma unroll
      for (int k = 0; k < NF; k++) acc[k] += dv * x[k];
    }
#pragma unroll
    for (int k = 0; k < NF; k++) div[k] = d == 0 ? acc[k] : div[k] + acc[k];
  }

  // C2: Fn - extrapolated normal flux at every (fpt, el), per flux point
  // or (PAIR) per line: one pass over a line's points gives both ends
  constexpr int NE = PAIR ? 2 : 1;  // flux points per work item
  for (int it = tid; act && it < (NFP / NE) * EB; it += NT) {
    const int l = it / EB, fe = it - (it / EB) * EB;
    const int ee = e0 + fe;
    const int pr = PAIR ? __ldg(&t.linePair[l]) : l;
    const int f0 = pr & 0xffff;
    const int base = __ldg(&t.fptBase[f0]), dn = __ldg(&t.fptDn[f0]);
    const int side0 = PAIR ? 0 : __ldg(&t.fptSide[f0]);
    const int stride = dn == 0 ? 1 : (dn == 1 ? N : N * N);
    R acc[NE][NF];
#pragma unroll
    for (int j = 0; j < NE; j++)
#pragma unroll
      for (int k = 0; k < NF; k++) acc[j][k] = R(0.0);
#pragma unroll
    for (int m = 0; m < N; m++) {
      const R *x = &sF[(dn * NS + base + m * stride) * ROW + fe * NF];
#pragma unroll
      for (int j = 0; j < NE; j++) {
        const R ev = sEF[(j ? 1 : side0) * N + m];
#pragma unroll
        for (int k = 0; k < NF; k++) acc[j][k] += ev * x[k];
      }
    }
    const bool v = fe < nValid;
#pragma unroll
    for (int j = 0; j < NE; j++) {
      const int f = j ? pr >> 16 : f0;
#pragma unroll
      for (int k = 0; k < NF; k++) {
        const R q = v ? a.Fn[((long long)f * E + ee) * NF + k] - acc[j][k] : R(0.0);
        sQ[f * ROW + fe * NF + k] = q;
        if (a.disFn_dbg && v) a.disFn_dbg[((long long)f * E + ee) * NF + k] = q;
      }
    }
  }
  __syncthreads();

  // D: correction and RK update at (s, el)
  if (valid) {
    R cq[NF];
#pragma unroll
    for (int k = 0; k < NF; k++) cq[k] = R(0.0);
#pragma unroll
    for (int fc = 0; fc < 2 * ND; fc++) {
      const int fp = __ldg(&t.corrFpt[s * 2 * ND + fc]);
      const R cv = __ldg(&t.corrVal[s * 2 * ND + fc]);
      const R *x = &sQ[fp * ROW + el * NF];
#pragma unroll
      for (int k = 0; k < NF; k++) cq[k] += cv * x[k];
    }
    const R rdJ = R(1.0) / a.detJ[(long long)s * E + e];  // one reciprocal per point
    const R dt = R(dtIn);
    const R rka = R(a.rka_next), rkb = R(a.rkb);
    const bool finalStage = a.mode == MODE_RK_FINAL || (a.mode == MODE_JAMESON && a.stage == a.nRK - 1);
#pragma unroll
    for (int k = 0; k < NF; k++) {
      const long long gi = ((long long)s * E + e) * NF + k;
      R dv = cq[k] + div[k];
      if (a.divF_out) a.divF_out[gi] = dv;
      if (a.mode == MODE_RESIDUAL) continue;
      if (a.src) dv = dv + a.src[gi];
      const R u = sU[s * ROW + el * NF + k];
      R unew;
      if constexpr (!F32) {
        if (a.mode == MODE_RK_STAGE) {
          const R u0 = a.stage == 0 ? u : a.U0[gi];
          if (a.stage == 0) a.U0[gi] = u;
          unew = u0 - rka * dv * rdJ * dt;
          const R base = a.stage == 0 ? u0 : a.acc[gi];
          a.acc[gi] = base - rkb * dv * rdJ * dt;
        } else if (a.mode == MODE_RK_FINAL) {
          const R base = a.nRK == 1 ? u : a.acc[gi];
          unew = base - rkb * dv * rdJ * dt;
        } else {
          const R u0 = a.stage == 0 ? u : a.U0[gi];
          if (a.stage == 0) a.U0[gi] = u;
          unew = u0 - rka * dv * rdJ * dt;
        }
      } else {
        // precision form: increments in acc, compensated final addition
        const R inc = dv * rdJ * dt;
        if (a.mode == MODE_RK_STAGE) {
          const R u0 = a.stage == 0 ? u : a.U0[gi];
          if (a.stage == 0) a.U0[gi] = u;
          unew = u0 - rka * inc;
          a.acc[gi] = (a.stage == 0 ? R(0) : a.acc[gi]) - rkb * inc;
        } else if (finalStage) {
          const bool fromU0 = (a.mode == MODE_RK_FINAL && a.nRK > 1) || (a.mode == MODE_JAMESON && a.stage > 0);
          const R u0 = fromU0 ? a.U0[gi] : u;
          const R sum = a.mode == MODE_RK_FINAL ? (a.nRK > 1 ? a.acc[gi] : R(0)) - rkb * inc : -(rka * inc);
          R c;
          two_sum_tp(u0, a.comp[gi] + sum, unew, c);
          a.comp[gi] = c;
        } else {
          const R u0 = a.stage == 0 ? u : a.U0[gi];
          if (a.stage == 0) a.U0[gi] = u;
          unew = u0 - rka * inc;
        }
      }
      a.Uout[gi] = unew;
      sU[s * ROW + el * NF + k] = unew;
    }
  }
  if (a.mode == MODE_RESIDUAL || !a.Ufpts_out) return;
  __syncthreads();

  // E: new state at the flux points (per flux point or, PAIR, per line)
  for (int it = tid; act && it < (NFP / NE) * EB; it += NT) {
    const int l = it / EB, fe = it - (it / EB) * EB;
    if (fe >= nValid) continue;
    const int ee = e0 + fe;
    const int pr = PAIR ? __ldg(&t.linePair[l]) : l;
    const int f0 = pr & 0xffff;
    const int base = __ldg(&t.fptBase[f0]), dn = __ldg(&t.fptDn[f0]);
    const int side0 = PAIR ? 0 : __ldg(&t.fptSide[f0]);
    const int stride = dn == 0 ? 1 : (dn == 1 ? N : N * N);
    R acc[NE][NF];
#pragma unroll
    for (int j = 0; j < NE; j++)
#pragma unroll
      for (int k = 0; k < NF; k++) acc[j][k] = R(0.0);
#pragma unroll
    for (int m = 0; m < N; m++) {
      const R *x = &sU[(base + m * stride) * ROW + fe * NF];
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
      for (int k = 0; k < NF; k++) a.Ufpts_out[((long long)f * E + ee) * NF + k] = acc[j][k];
    }
  }
}

template <int ND, int P, bool VISC, typename R>
__global__ void __launch_bounds__(Tp<ND, P, R>::NT) k_elem_tp(ElemArgsT<R> a, TpTablesT<R> t) {
  pdl_wait();
  pdl_trigger();
  extern __shared__ __align__(16) unsigned char smem_bytes[];
  elem_tp_block<ND, P, VISC, R>(a, t, blockIdx.x, smem_bytes);
}

constexpr int kMultiNT = 256;  // threads of a many-order CTA: at least every order's NT
static_assert(Tp<2, 0>::NT <= kMultiNT && Tp<2, 5>::NT <= kMultiNT && Tp<3, 3>::NT <= kMultiNT &&
                  Tp<3, 5>::NT <= kMultiNT && Tp<2, 2, float>::NT <= kMultiNT,
              "a tensor-product block exceeds the many-order CTA");

// the arguments travel as one kernel parameter (above the classic 4 KB,
// within the 32,764 bytes sm_70+ take since CUDA 12.1)
static_assert(sizeof(MultiElemArgsT<double>) < 32000, "many-order arguments exceed the kernel parameter space");

template <int ND, typename R>
__global__ void __launch_bounds__(kMultiNT) k_elem_multi(const __grid_constant__ MultiElemArgsT<R> m) {
  pdl_wait();
  pdl_trigger();
  extern __shared__ __align__(16) unsigned char smem_bytes[];
  __shared__ int item;
  for (;;) {
    if (threadIdx.x == 0) item = (int)atomicAdd(m.next, 1u);
    __syncthreads();
    const int w = item;
    __syncthreads();  // every thread has the item before thread 0 takes the next
    if (w >= m.total) break;
    int g = 0;
    while (g + 1 < m.nGroups && w >= m.start[g + 1]) g++;
    const int blk = w - m.start[g];
    switch (m.order[g]) {
      case 0: elem_tp_block<ND, 0, false, R, false>(m.a[g], m.t[g], blk, smem_bytes); break;
      case 1: elem_tp_block<ND, 1, false, R, false>(m.a[g], m.t[g], blk, smem_bytes); break;
      case 2: elem_tp_block<ND, 2, false, R, false>(m.a[g], m.t[g], blk, smem_bytes); break;
      case 3: elem_tp_block<ND, 3, false, R, false>(m.a[g], m.t[g], blk, smem_bytes); break;
      case 4: elem_tp_block<ND, 4, false, R, false>(m.a[g], m.t[g], blk, smem_bytes); break;
      default: elem_tp_block<ND, 5, false, R, false>(m.a[g], m.t[g], blk, smem_bytes); break;
    }
    __syncthreads();  // the next block reuses the shared memory
  }
  // the last CTA out resets the counters for the next launch (all CTAs have
  // taken their last item by then) and, after a step's last stage, advances
  // the time of every group
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(m.done, 1u) == gridDim.x - 1) {
      *m.next = 0u;
      *m.done = 0u;
      if (m.finalStage)
        for (int g = 0; g < m.nGroups; g++) *m.timeAcc[g] += *m.a[g].dt;
      __threadfence();
    }
  }
}

template <int ND, typename R>
size_t multi_smem(const MultiElemArgsT<R> &m) {
  size_t b = 0;
  for (int g = 0; g < m.nGroups; g++) {
    size_t x = 0;
    switch (m.order[g]) {
      case 0: x = Tp<ND, 0, R>::SMEM; break;
      case 1: x = Tp<ND, 1, R>::SMEM; break;
      case 2: x = Tp<ND, 2, R>::SMEM; break;
      case 3: x = Tp<ND, 3, R>::SMEM; break;
      case 4: x = Tp<ND, 4, R>::SMEM; break;
      default: x = Tp<ND, 5, R>::SMEM; break;
    }
    b = x > b ? x : b;
  }
  return b;
}

// the largest block's shared memory over all orders (the attribute is set
// once per device, whichever orders a batch holds)
template <int ND, typename R>
constexpr size_t multi_smem_max() {
  size_t b = Tp<ND, 0, R>::SMEM;
  b = Tp<ND, 1, R>::SMEM > b ? Tp<ND, 1, R>::SMEM : b;
  b = Tp<ND, 2, R>::SMEM > b ? Tp<ND, 2, R>::SMEM : b;
  b = Tp<ND, 3, R>::SMEM > b ? Tp<ND, 3, R>::SMEM : b;
  b = Tp<ND, 4, R>::SMEM > b ? Tp<ND, 4, R>::SMEM : b;
  b = Tp<ND, 5, R>::SMEM > b ? Tp<ND, 5, R>::SMEM : b;
  return b;
}

template <int ND, typename R>
void launch_multi(const MultiElemArgsT<R> &m, cudaStream_t st) {
  const int smem = (int)multi_smem<ND, R>(m);
  static std::atomic<unsigned long long> attrDev{0};
  smem_attr(k_elem_multi<ND, R>, (int)multi_smem_max<ND, R>(), attrDev);
  int per = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_elem_multi<ND, R>, kMultiNT, smem);
  const int g = std::max(1, std::min(m.total, std::max(per, 1) * sm_count(current_device())));
  launch_k(k_elem_multi<ND, R>, g, kMultiNT, smem, st, m);
}

template <int ND, int P, typename R, bool VISC = false>
void launch_tp(const ElemArgsT<R> &a, const TpTablesT<R> &t, cudaStream_t st) {
  using T = Tp<ND, P, R>;
  static std::atomic<unsigned long long> attrDev{0};
  smem_attr(k_elem_tp<ND, P, VISC, R>, (int)T::SMEM, attrDev);
  int g = (a.E + T::EB - 1) / T::EB;
  launch_k(k_elem_tp<ND, P, VISC, R>, g, T::NT, T::SMEM, st, a, t);
}

#define FR_TP_ORDERS(X) X(2, 0) X(2, 1) X(2, 2) X(2, 3) X(2, 4) X(2, 5) X(3, 0) X(3, 1) X(3, 2) X(3, 3) X(3, 4) X(3, 5)

}  // namespace

bool tp_supported(int nDims, int order) { return (nDims == 2 || nDims == 3) && order >= 0 && order <= 5; }

template <typename R>
int tp_elems_per_block(int nDims, int order) {
#define FR_TP_EB(ND, P) \
  if (nDims == ND && order == P) return Tp<ND, P, R>::EB;
  FR_TP_ORDERS(FR_TP_EB)
#undef FR_TP_EB
  return 0;
}

template <typename R>
void launch_element_stage_tp(int nDims, int order, const ElemArgsT<R> &a, const TpTablesT<R> &t, cudaStream_t st) {
  if (a.E <= 0) return;
#define FR_TP_CASE(ND, P) \
  if (nDims == ND && order == P) return launch_tp<ND, P, R>(a, t, st);
  FR_TP_ORDERS(FR_TP_CASE)
#undef FR_TP_CASE
}

template <typename R>
void launch_element_stage_tp_visc(int nDims, int order, const ElemArgsT<R> &a, const TpTablesT<R> &t,
                                  cudaStream_t st) {
  if (a.E <= 0) return;
#define FR_TPV_CASE(ND, P) \
  if (nDims == ND && order == P) return launch_tp<ND, P, R, true>(a, t, st);
  FR_TP_ORDERS(FR_TPV_CASE)
#undef FR_TPV_CASE
}

template <typename R>
void launch_element_stage_multi(int nDims, const MultiElemArgsT<R> &m, cudaStream_t st) {
  if (m.total <= 0) return;
  if (nDims == 2)
    launch_multi<2, R>(m, st);
  else
    launch_multi<3, R>(m, st);
}
template void launch_element_stage_multi<double>(int, const MultiElemArgsT<double> &, cudaStream_t);
template void launch_element_stage_multi<float>(int, const MultiElemArgsT<float> &, cudaStream_t);

template int tp_elems_per_block<double>(int, int);
template int tp_elems_per_block<float>(int, int);
template void launch_element_stage_tp<double>(int, int, const ElemArgsT<double> &, const TpTablesT<double> &,
                                              cudaStream_t);
template void launch_element_stage_tp<float>(int, int, const ElemArgsT<float> &, const TpTablesT<float> &,
                                             cudaStream_t);
template void launch_element_stage_tp_visc<double>(int, int, const ElemArgsT<double> &, const TpTablesT<double> &,
                                                   cudaStream_t);
template void launch_element_stage_tp_visc<float>(int, int, const ElemArgsT<float> &, const TpTablesT<float> &,
                                                  cudaStream_t);

}  // namespace frk
