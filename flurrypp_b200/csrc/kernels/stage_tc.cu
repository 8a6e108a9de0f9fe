// Element stage of the precision form on the 5th-generation tensor cores
// (2-D orders 1..4, 3-D order 1).
//
// The same stage as k_elem_tma (flux, divergence, extrapolated normal flux,
// correction, RK update, extrapolation to the flux points; reference:
// solver.cpp:470-572, 707-736, 906-1058) with the operators applied as the
// reference applies them, dense matrices, but as tcgen05.mma kind::tf32
// contractions with FP32 accumulation in tensor memory.  Each operand is
// split x = hi + lo into two TF32 values and a product is formed from
// hi*hi + hi*lo + lo*hi (3xTF32: ~2^-22 relative, FP32-like).
//
// One CTA holds EB elements (2-D: 32 x 4 fields; 3-D: 24 x 5 fields, the
// last 8 rows padding); the (element, field) columns of a tile are the rows
// of every MMA (M = 128, one TMEM lane each), so with the element tile as
// the A operand and an operator as the B operand:
//   GEMM1  D[:, 0:NSp | NSp:NSp+NFPp] = F^T [128 x ND*NS] * [grad_d ... ; extFn_d ...]^T
//          (divergence and extrapolated normal flux in one MMA chain)
//   GEMM2  D[:, 0:NSp] += (Fn - disFn)^T [128 x NFP] * corr^T
//   GEMM3  D[:, NSp:]   = U_new^T [128 x NS] * ext^T
// The A operands are written by the threads that compute them, straight into
// the K-major no-swizzle canonical layout (8-row x 16-byte core matrices);
// the operators are packed in that layout on the host.  Tiles move by TMA as
// in k_elem_tma (same tensor maps, EB-element boxes).  2-D orders 1..4 and
// 3-D order 1: the split dense operators and the A operands of larger orders
// do not fit next to the tiles in shared memory (3-D P2: 287 KB of 227).
#include <cmath>
#include <cstring>
#include <vector>

#include "launch.cuh"
#include "stage.hpp"
#include "umma.cuh"

namespace frk {

namespace {

constexpr int r8(int x) { return (x + 7) / 8 * 8; }
constexpr int r16(int x) { return (x + 15) / 16 * 16; }
constexpr int cmax(int a, int b) { return a > b ? a : b; }

template <int ND, int P>
struct Tc {
  static constexpr int N = P + 1, NS = ND == 2 ? N * N : N * N * N, NFP = 2 * ND * (ND == 2 ? N : N * N);
  static constexpr int NF = ND + 2, EB = ND == 2 ? 32 : 24, M = 128, NT = 128;
  static constexpr int ROW = EB * NF;  // values per point row of a tile: 128 (2-D), 120 (3-D)
  static constexpr int NSp = r16(NS), NFPp = r16(NFP), N1 = NSp + NFPp;
  static constexpr int K1p = r8(ND * NS), K2p = r8(NFP), K3p = r8(NS);
  static constexpr int KAp = cmax(K1p, cmax(K2p, K3p));
  static constexpr int SB1 = N1 * K1p, SB2 = NSp * K2p, SB3 = NFPp * K3p;
  static constexpr int O_B1H = 0, O_B1L = SB1, O_B2H = 2 * SB1, O_B2L = 2 * SB1 + SB2;
  static constexpr int O_B3H = 2 * SB1 + 2 * SB2, O_B3L = O_B3H + SB3;
  static constexpr int OPS = 2 * (SB1 + SB2 + SB3);
  static constexpr int TCOLS = N1 <= 32 ? 32 : (N1 <= 64 ? 64 : 128);
  static constexpr int al(int n) { return (n + 31) / 32 * 32; }  // floats, 128 bytes
  static constexpr int O_OPS = 0;
  static constexpr int O_AH = O_OPS + al(OPS);
  static constexpr int O_AL = O_AH + al(M * KAp);
  static constexpr int O_U = O_AL + al(M * KAp);
  static constexpr int O_U0 = O_U + al(NS * ROW);
  static constexpr int O_ACC = O_U0 + al(NS * ROW);
  static constexpr int O_CMP = O_ACC + al(NS * ROW);
  static constexpr int O_FN = O_CMP + al(NS * ROW);
  static constexpr int O_J = O_FN + al(NFP * ROW);
  static constexpr int O_DET = O_J + al(ND * NS * EB * ND);
  static constexpr int O_BAR = O_DET + al(NS * EB);
  static constexpr size_t SMEM = 4 * (size_t)(O_BAR + 32) + 128;
  static_assert(SMEM <= 227 * 1024, "tensor-core tile set does not fit in shared memory");
  static_assert(N1 <= 256 && N1 % 16 == 0, "MMA N");
  static_assert(ROW <= M, "element tile rows exceed the MMA rows");
};

// float offset of (row r, column k) in a K-major no-swizzle operand whose K
// extent is Kp: core matrix (r/8, k/4) of 32 floats, K chunks adjacent
// (128 bytes apart), row groups Kp*8 floats apart
__host__ __device__ constexpr int blk(int r, int k, int Kp) {
  return (r >> 3) * (Kp * 8) + (k >> 2) * 32 + (r & 7) * 4 + (k & 3);
}

__device__ __forceinline__ uint64_t desc_at(const float *base, int t, int Kp) {
  return umma_desc_kmajor(smem_u32(base) + 256u * t, 128u, (uint32_t)Kp * 32u);
}

// One contraction D (+)= A * B^T with 3xTF32 terms, K in steps of 8.
__device__ __forceinline__ void gemm3x(uint32_t d, const float *aH, const float *aL, const float *bH,
                                       const float *bL, int Kp, uint32_t idesc, bool accumulate) {
  for (int t = 0; t < Kp / 8; t++) {
    umma_tf32(d, desc_at(aL, t, Kp), desc_at(bH, t, Kp), idesc, accumulate || t > 0);
    umma_tf32(d, desc_at(aH, t, Kp), desc_at(bL, t, Kp), idesc, true);
    umma_tf32(d, desc_at(aH, t, Kp), desc_at(bH, t, Kp), idesc, true);
  }
}

__device__ __forceinline__ void split_store(float *aH, float *aL, int idx, float x) {
  const float h = tf32_rna(x);
  aH[idx] = h;
  aL[idx] = tf32_rna(x - h);
}

__device__ __forceinline__ void two_sum_tc(float a, float b, float &s, float &e) {
  s = __fadd_rn(a, b);
  const float bb = __fsub_rn(s, a);
  e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bb)), __fsub_rn(b, bb));
}

constexpr uint32_t kWait = 1u << 22;

template <int ND, int P>
__global__ void __launch_bounds__(128) k_elem_tc(ElemArgsT<float> a, const float *__restrict__ ops,
                                                 const __grid_constant__ TmaMaps mp) {
  pdl_wait();
  pdl_trigger();
  using T = Tc<ND, P>;
  constexpr int NS = T::NS, NFP = T::NFP, NF = T::NF, EB = T::EB, ROW = T::ROW;
  constexpr int NSp = T::NSp, K1p = T::K1p, K2p = T::K2p, K3p = T::K3p;
  extern __shared__ __align__(128) unsigned char smem_bytes[];
  float *sm = reinterpret_cast<float *>((reinterpret_cast<uintptr_t>(smem_bytes) + 127) & ~uintptr_t(127));
  float *sOps = sm + T::O_OPS;
  float *sAh = sm + T::O_AH, *sAl = sm + T::O_AL;
  float *sU = sm + T::O_U, *sU0 = sm + T::O_U0, *sAcc = sm + T::O_ACC, *sCmp = sm + T::O_CMP;
  float *sFn = sm + T::O_FN, *sJ = sm + T::O_J, *sDet = sm + T::O_DET;
  uint64_t *bar = reinterpret_cast<uint64_t *>(sm + T::O_BAR);  // tiles A, tiles B, MMA
  uint32_t *tslot = reinterpret_cast<uint32_t *>(bar + 3);

  const int tid = threadIdx.x, warp = tid >> 5;
  const int E = a.E, e0 = blockIdx.x * EB;
  const int nValid = min(EB, E - e0);
  const int r = tid;                 // this thread's MMA row / TMEM lane: (element r/NF, field r%NF)
  const int re = r / NF;
  const bool rrow = r < ROW;         // rows ROW..127 (3-D) are padding: zero A rows, no tile access
  const bool rvalid = rrow && re < nValid;

  const bool finalStage = a.mode == MODE_RK_FINAL || (a.mode == MODE_JAMESON && a.stage == a.nRK - 1);
  const bool needU0 = ((a.mode == MODE_RK_STAGE || a.mode == MODE_JAMESON) && a.stage > 0) ||
                      (a.mode == MODE_RK_FINAL && a.nRK > 1);
  const bool needAcc = (a.mode == MODE_RK_STAGE && a.stage > 0) || (a.mode == MODE_RK_FINAL && a.nRK > 1);
  const bool needCmp = finalStage;
  const bool needDet = a.mode != MODE_RESIDUAL;
  const double dtIn = a.mode == MODE_RESIDUAL ? 0.0 : (a.eleDt ? (rvalid ? a.eleDt[e0 + re] : 0.0) : *a.dt);

  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_init(&bar[2], 1);
    fence_mbar_init();
  }
  if (warp == 0) tmem_alloc(tslot, T::TCOLS);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = *tslot;
  const uint32_t tlane = tbase + ((uint32_t)(warp * 32) << 16);

  if (tid == 0) {
    mbar_arrive_expect_tx(&bar[0], 4u * (NS * ROW + ND * NS * EB * ND));
    tma_load_2d(sU, &mp.U, e0 * NF, 0, &bar[0]);
    tma_load_3d(sJ, &mp.J, e0 * ND, 0, 0, &bar[0]);
    uint32_t bytes = 4u * NFP * ROW;
    if (needU0) bytes += 4u * NS * ROW;
    if (needAcc) bytes += 4u * NS * ROW;
    if (needCmp) bytes += 4u * NS * ROW;
    if (needDet) bytes += 4u * NS * EB;
    mbar_arrive_expect_tx(&bar[1], bytes);
    tma_load_2d(sFn, &mp.Fn, e0 * NF, 0, &bar[1]);
    if (needU0) tma_load_2d(sU0, &mp.U0, e0 * NF, 0, &bar[1]);
    if (needAcc) tma_load_2d(sAcc, &mp.acc, e0 * NF, 0, &bar[1]);
    if (needCmp) tma_load_2d(sCmp, &mp.comp, e0 * NF, 0, &bar[1]);
    if (needDet) tma_load_2d(sDet, &mp.det, e0, 0, &bar[1]);
  }
  // operators (packed on the host in the MMA layout), and the zero padding
  // columns of the first A operand
  for (int i = tid; i < T::OPS / 4; i += 128)
    reinterpret_cast<float4 *>(sOps)[i] = reinterpret_cast<const float4 *>(ops)[i];
  constexpr int PAD1 = K1p - ND * NS;
  if constexpr (PAD1 > 0) {
    for (int i = tid; i < 128 * PAD1; i += 128) {
      const int rr = i / PAD1, k = ND * NS + i % PAD1;
      sAh[blk(rr, k, K1p)] = 0.0f;
      sAl[blk(rr, k, K1p)] = 0.0f;
    }
  }
  // padding rows of the first A operand (the flux loop writes rows < ROW)
  if constexpr (ROW < 128) {
    for (int i = tid; i < (128 - ROW) * ND * NS; i += 128) {
      const int rr = ROW + i / (ND * NS), k = i % (ND * NS);
      sAh[blk(rr, k, K1p)] = 0.0f;
      sAl[blk(rr, k, K1p)] = 0.0f;
    }
  }

  bool ok = __syncthreads_and(mbar_wait_bounded(&bar[0], 0, kWait));
  uint32_t mmaPhase = 0;
  if (ok) {
    if ((a.mode == MODE_RK_STAGE || a.mode == MODE_JAMESON) && a.stage == 0 && tid == 0) {
      tma_store_2d(&mp.U0, e0 * NF, 0, sU);
      tma_commit();
    }
    // flux at (s, el): reference-space F_d into the A operand, column d*NS + s
    for (int it = tid; it < NS * EB; it += 128) {
      const int s = it / EB, el = it - (it / EB) * EB;
      float Fp[ND][NF];
      if (el < nValid) {
        inviscid_flux<ND, float>(&sU[s * ROW + el * NF], Fp, float(a.gamma));
      } else {
#pragma unroll
        for (int d = 0; d < ND; d++)
#pragma unroll
          for (int k = 0; k < NF; k++) Fp[d][k] = 0.0f;
      }
#pragma unroll
      for (int d1 = 0; d1 < ND; d1++) {
        const float *Jr = &sJ[(d1 * NS + s) * EB * ND + el * ND];
#pragma unroll
        for (int k = 0; k < NF; k++) {
          float f = 0.0f;
#pragma unroll
          for (int d2 = 0; d2 < ND; d2++) f += Jr[d2] * Fp[d2][k];
          split_store(sAh, sAl, blk(el * NF + k, d1 * NS + s, K1p), f);
          if (a.F_dbg && el < nValid) a.F_dbg[(((long long)d1 * NS + s) * E + e0 + el) * NF + k] = f;
        }
      }
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (tid == 0) {
      gemm3x(tbase, sAh, sAl, sOps + T::O_B1H, sOps + T::O_B1L, K1p, umma_idesc_tf32(128, T::N1), false);
      umma_commit(&bar[2]);
    }
    ok = __syncthreads_and(mbar_wait_bounded(&bar[2], mmaPhase, kWait) && mbar_wait_bounded(&bar[1], 0, kWait));
    mmaPhase ^= 1;
  }
  if (ok) {
    tc_fence_after();
    // Fn - extrapolated normal flux (TMEM columns NSp ..) -> second A operand
    for (int c = 0; c < NFP; c += 8) {
      float v[8];
      tmem_ld8(tlane + NSp + c, v);
#pragma unroll
      for (int i = 0; i < 8; i++) {
        const int f = c + i;
        if (f < NFP) {
          const float q = rrow ? sFn[f * ROW + r] - v[i] : 0.0f;
          split_store(sAh, sAl, blk(r, f, K2p), q);
          if (a.disFn_dbg && rvalid) a.disFn_dbg[((long long)f * E + e0) * NF + r] = q;
        } else if (f < K2p) {
          sAh[blk(r, f, K2p)] = 0.0f;
          sAl[blk(r, f, K2p)] = 0.0f;
        }
      }
    }
    for (int f = (NFP + 7) / 8 * 8; f < K2p; f++) {
      sAh[blk(r, f, K2p)] = 0.0f;
      sAl[blk(r, f, K2p)] = 0.0f;
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (tid == 0) {
      gemm3x(tbase, sAh, sAl, sOps + T::O_B2H, sOps + T::O_B2L, K2p, umma_idesc_tf32(128, NSp), true);
      umma_commit(&bar[2]);
      tma_wait_read_all();  // the stage-0 U0 store has read sU
    }
    ok = __syncthreads_and(mbar_wait_bounded(&bar[2], mmaPhase, kWait));
    mmaPhase ^= 1;
  }
  if (ok) {
    tc_fence_after();
    // divergence + correction (TMEM columns 0 ..): RK update, new state into
    // the tiles and into the third A operand
    const float dt = float(dtIn);
    const float rka = float(a.rka_next), rkb = float(a.rkb);
    for (int c = 0; c < NS; c += 8) {
      float v[8];
      tmem_ld8(tlane + c, v);
#pragma unroll
      for (int i = 0; i < 8; i++) {
        const int s = c + i;
        if (s >= NS) break;
        if (!rrow) {  // padding row: a zero row of the third A operand
          sAh[blk(r, s, K3p)] = 0.0f;
          sAl[blk(r, s, K3p)] = 0.0f;
          continue;
        }
        const int li = s * ROW + r;
        const long long gi = ((long long)s * E + e0) * NF + r;
        float dv = v[i];
        if (a.divF_out && rvalid) a.divF_out[gi] = dv;
        if (a.mode == MODE_RESIDUAL) continue;
        if (a.src && rvalid) dv = dv + a.src[gi];
        const float rdJ = 1.0f / sDet[s * EB + re];
        const float inc = dv * rdJ * dt;
        const float u = sU[li];
        float unew;
        if (a.mode == MODE_RK_STAGE) {
          const float u0 = a.stage == 0 ? u : sU0[li];
          unew = u0 - rka * inc;
          sAcc[li] = (a.stage == 0 ? 0.0f : sAcc[li]) - rkb * inc;
        } else if (finalStage) {
          const float u0 = (a.mode == MODE_RK_FINAL && a.nRK > 1) || (a.mode == MODE_JAMESON && a.stage > 0) ? sU0[li] : u;
          const float sum = a.mode == MODE_RK_FINAL ? (a.nRK > 1 ? sAcc[li] : 0.0f) - rkb * inc : -(rka * inc);
          float cc;
          two_sum_tc(u0, sCmp[li] + sum, unew, cc);
          sCmp[li] = cc;
        } else {
          const float u0 = a.stage == 0 ? u : sU0[li];
          unew = u0 - rka * inc;
        }
        sU[li] = unew;
        split_store(sAh, sAl, blk(r, s, K3p), unew);
      }
    }
    for (int s = NS; s < K3p; s++) {
      sAh[blk(r, s, K3p)] = 0.0f;
      sAl[blk(r, s, K3p)] = 0.0f;
    }
    const bool more = a.mode != MODE_RESIDUAL;
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (more && tid == 0) {
      tma_store_2d(&mp.U, e0 * NF, 0, sU);
      if (a.mode == MODE_RK_STAGE) tma_store_2d(&mp.acc, e0 * NF, 0, sAcc);
      if (needCmp) tma_store_2d(&mp.comp, e0 * NF, 0, sCmp);
      tma_commit();
      if (a.Ufpts_out) {
        gemm3x(tbase + NSp, sAh, sAl, sOps + T::O_B3H, sOps + T::O_B3L, K3p, umma_idesc_tf32(128, T::NFPp), false);
        umma_commit(&bar[2]);
      }
    }
    if (more && a.Ufpts_out) {
      ok = __syncthreads_and(mbar_wait_bounded(&bar[2], mmaPhase, kWait));
      mmaPhase ^= 1;
      if (ok) {
        tc_fence_after();
        // new state at the flux points (TMEM columns NSp ..) -> the Fn tile -> TMA store
        for (int c = 0; c < NFP; c += 8) {
          float v[8];
          tmem_ld8(tlane + NSp + c, v);
#pragma unroll
          for (int i = 0; i < 8; i++)
            if (c + i < NFP && rrow) sFn[(c + i) * ROW + r] = v[i];
        }
        fence_async_smem();
        __syncthreads();
        if (tid == 0) {
          tma_store_2d(&mp.Ufpts, e0 * NF, 0, sFn);
          tma_commit();
        }
      }
    }
  }
  if (!ok) {
    // a bounded wait ran out: flag it and let copies and MMAs in flight end
    // (bounded) before the tensor memory is released; the MMA phase last
    // waited for has the parity before the flip
    if (tid == 0 && a.err) atomicOr(a.err, 1);
    mbar_wait_bounded(&bar[0], 0, kWait);
    mbar_wait_bounded(&bar[1], 0, kWait);
    mbar_wait_bounded(&bar[2], mmaPhase ^ 1u, kWait);
  }
  if (tid == 0) tma_wait_read_all();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tmem_dealloc(tbase, T::TCOLS);
}

template <int ND, int P>
void launch_tc(const ElemArgsT<float> &a, const float *ops, const TmaMaps &m, cudaStream_t st) {
  using T = Tc<ND, P>;
  static std::atomic<unsigned long long> attrDev{0};
  smem_attr(k_elem_tc<ND, P>, (int)T::SMEM, attrDev);
  launch_k(k_elem_tc<ND, P>, (a.E + T::EB - 1) / T::EB, T::NT, T::SMEM, st, a, ops, m);
}

// host TF32 rounding, nearest with ties away from zero (as cvt.rna), low 13
// bits cleared
float tf32_host(double x) {
  float f = (float)x;
  uint32_t u;
  std::memcpy(&u, &f, 4);
  if ((u & 0x7F800000u) != 0x7F800000u) u = (u + 0x1000u) & 0xFFFFE000u;
  std::memcpy(&f, &u, 4);
  return f;
}

template <int ND, int P>
void pack(const double *const grad[3], const double *const extFn[3], const double *corr, const double *ext,
          std::vector<float> &blob) {
  using T = Tc<ND, P>;
  constexpr int NS = T::NS, NFP = T::NFP;
  blob.assign(T::OPS, 0.0f);
  auto put = [&](int oH, int oL, int row, int k, int Kp, double x) {
    const float h = tf32_host(x);
    blob[oH + blk(row, k, Kp)] = h;
    blob[oL + blk(row, k, Kp)] = tf32_host(x - (double)h);
  };
  for (int d = 0; d < ND; d++)
    for (int s = 0; s < NS; s++) {
      for (int n = 0; n < NS; n++) put(T::O_B1H, T::O_B1L, n, d * NS + s, T::K1p, grad[d][(size_t)n * NS + s]);
      for (int f = 0; f < NFP; f++)
        put(T::O_B1H, T::O_B1L, T::NSp + f, d * NS + s, T::K1p, extFn[d][(size_t)f * NS + s]);
    }
  for (int n = 0; n < NS; n++)
    for (int f = 0; f < NFP; f++) put(T::O_B2H, T::O_B2L, n, f, T::K2p, corr[(size_t)n * NFP + f]);
  for (int f = 0; f < NFP; f++)
    for (int s = 0; s < NS; s++) put(T::O_B3H, T::O_B3L, f, s, T::K3p, ext[(size_t)f * NS + s]);
}

}  // namespace

bool tc_supported(int nDims, int order) {
  return (nDims == 2 && order >= 1 && order <= 4) || (nDims == 3 && order == 1);
}

int tc_elems_per_block(int nDims, int order) {
  return tc_supported(nDims, order) ? (nDims == 2 ? Tc<2, 1>::EB : Tc<3, 1>::EB) : 0;
}

bool tc_pack_ops(int nDims, int order, const double *const grad[3], const double *const extFn[3],
                 const double *corr, const double *ext, std::vector<float> &blob) {
  if (nDims == 3) {
    if (order != 1) return false;
    pack<3, 1>(grad, extFn, corr, ext, blob);
    return true;
  }
  switch (order) {
    case 1: pack<2, 1>(grad, extFn, corr, ext, blob); return true;
    case 2: pack<2, 2>(grad, extFn, corr, ext, blob); return true;
    case 3: pack<2, 3>(grad, extFn, corr, ext, blob); return true;
    case 4: pack<2, 4>(grad, extFn, corr, ext, blob); return true;
    default: return false;
  }
}

size_t tc_smem_bytes(int nDims, int order) {
  if (nDims == 3) return order == 1 ? Tc<3, 1>::SMEM : 0;
  switch (order) {
    case 1: return Tc<2, 1>::SMEM;
    case 2: return Tc<2, 2>::SMEM;
    case 3: return Tc<2, 3>::SMEM;
    case 4: return Tc<2, 4>::SMEM;
    default: return 0;
  }
}

void launch_element_stage_tc(int nDims, int order, const ElemArgsT<float> &a, const float *ops, const TmaMaps &m,
                             cudaStream_t st) {
  if (a.E <= 0) return;
  if (nDims == 3) {
    if (order == 1) launch_tc<3, 1>(a, ops, m, st);
    return;
  }
  switch (order) {
    case 1: return launch_tc<2, 1>(a, ops, m, st);
    case 2: return launch_tc<2, 2>(a, ops, m, st);
    case 3: return launch_tc<2, 3>(a, ops, m, st);
    case 4: return launch_tc<2, 4>(a, ops, m, st);
    default: return;
  }
}

}  // namespace frk
