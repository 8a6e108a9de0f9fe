// Launch interface of the per-stage FR kernels (FP64 plain form).
// All arrays are device pointers in the reference layout
// ([point][element][field], last index fastest).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include "fr_physics.cuh"

namespace frk {

// A dense operator matrix stored by its nonzero entries (row-compressed).
// Applying it is the reference's cblas_dgemm on the same matrix with the
// exact zeros skipped: each output is the same dot product over the nonzero
// terms (a zero term adds +-0 and changes no sum).
struct Csr {
  int nRows = 0, nCols = 0;
  const int *rowptr = nullptr;
  const int *col = nullptr;
  const double *val = nullptr;
};

// out[r][n] = alpha * sum_c A[r][c] in[c][n] + beta * out[r][n], n < N.
void launch_apply_op(const Csr &A, const double *in, double *out, long long N, double alpha,
                     double beta, cudaStream_t st);

// Face-point table, one entry per flux point of each face, sorted by left slot.
struct FaceTable {
  int n = 0;
  int nInterior = 0;            // interior points first, then boundary points
  const int *slotL = nullptr;   // fpt*E + e of the left side
  const int *slotR = nullptr;   // fpt*E + e of the right side, or -(bc+2) on a boundary
  const double *nrm = nullptr;  // [n][nDims] left unit normal
  const double *dAL = nullptr;
  const double *dAR = nullptr;
};

// Common inviscid flux on every face point: Fn_fpts at both sides and the
// left-side wave speed (reference: solver.cpp:752-758, face.cpp:163-208).
// Interior and boundary points run as two kernels (no BC code in the
// interior one).
void launch_faces_inviscid(int nDims, const FaceTable &ft, const double *Ufpts, double *Fn,
                           double *waveSp, const Phys &ph, cudaStream_t st);

enum ElemMode : int {
  MODE_RESIDUAL = 0,  // calcResidual only: divF -> divF_out
  MODE_RK_STAGE = 1,  // standard RK intermediate stage (timeStepA + running timeStepB)
  MODE_RK_FINAL = 2,  // standard RK final stage (remaining timeStepB)
  MODE_JAMESON = 3    // Jameson-form stage: U = U0 - RKa[s+1] divF/detJ dt
};

struct ElemArgs {
  int E = 0, nS = 0, nFp = 0, EB = 1;
  const double *U = nullptr;       // current stage state [nS][E][nF]
  const double *JGinv = nullptr;   // [nDims][nS][E][nDims]
  const double *detJ = nullptr;    // [nS][E]
  const double *Fn = nullptr;      // common normal flux * dA [nFp][E][nF]
  Csr grad[3], extFn[3], corr, ext;
  int mode = MODE_RESIDUAL;
  int stage = 0;
  int nRK = 4;
  double rka_next = 0.0, rkb = 0.0;
  const double *dt = nullptr;      // device scalar
  const double *eleDt = nullptr;   // per-element dt (dtType 2) or null
  const double *src = nullptr;     // P-multigrid source or null
  double *U0 = nullptr;            // RK base state (written at stage 0)
  double *acc = nullptr;           // running final-stage sum
  double *Uout = nullptr;          // next state
  double *divF_out = nullptr;      // optional divF of this stage
  double *Ufpts_out = nullptr;     // optional: next state at flux points
  double *F_dbg = nullptr;         // optional: F_spts [nDims][nS][E][nF]
  double *disFn_dbg = nullptr;     // optional: Fn - extrapolated flux [nFp][E][nF]
  unsigned int *err = nullptr;     // device status word (bit 0: a bounded wait ran out)
  double gamma = 1.4;
  // viscous stages: physical gradient at the solution points
  // [nDims][nS][E][nF] (stride between dimensions dUsStride), and constants
  const double *dUs = nullptr;
  long long dUsStride = 0;
  Phys ph{};
};

size_t elem_smem_bytes(int nDims, int nS, int nFp, int EB);
void launch_element_stage(int nDims, const ElemArgs &a, cudaStream_t st);

// Tensor-product form of the same operators (quads/hexes): the dense
// matrices' nonzeros, verified bitwise on the host, as 1-D tables.
//   grad_d[s][c] = D[i_d(s)][m]   for c on the line through s along d
//   ext[f][s]    = E1[side(f)][m] for s on the line of f (normal dim dn(f))
//   extFn_dn     = (side ? +1 : -1) * ext
//   corr[s][f]   = corrVal[s][face] at f = corrFpt[s][face], one per face
struct TpTables {
  const double *D = nullptr;        // [n][n]
  const double *E1 = nullptr;       // [2][n]   side 0: xi=-1, side 1: xi=+1
  const double *EFn1 = nullptr;     // [2][n]   E1 times the reference normal
  const int *fptBase = nullptr;     // [nFp] first solution point of the line
  const int *fptDn = nullptr;       // [nFp] normal dimension
  const int *fptSide = nullptr;     // [nFp]
  const int *corrFpt = nullptr;     // [nS][2*nDims]
  const double *corrVal = nullptr;  // [nS][2*nDims]
};
bool tp_supported(int nDims, int order);

// TMA descriptors of the tiles the TMA element kernel moves (one row block of
// points x EB elements of the reference layout per copy).
struct TmaMaps {
  CUtensorMap U;      // [nS][E*nF]    load + store (in place)
  CUtensorMap U0;     // [nS][E*nF]
  CUtensorMap acc;    // [nS][E*nF]
  CUtensorMap Fn;     // [nFp][E*nF]
  CUtensorMap Ufpts;  // [nFp][E*nF]   store
  CUtensorMap J;      // [nDims][nS][E*nDims]
  CUtensorMap det;    // [nS][E]
};
int tma_elems_per_block(int nDims, int order);
size_t tma_smem_bytes(int nDims, int order);
void launch_element_stage_tma(int nDims, int order, const ElemArgs &a, const TpTables &t,
                              const TmaMaps &m, cudaStream_t st);
int tp_elems_per_block(int nDims, int order);
void launch_element_stage_tp(int nDims, int order, const ElemArgs &a, const TpTables &t,
                             cudaStream_t st);

// Viscous (LDG) stage pieces (kernels/stage_visc_fp64.cu).
struct GradArgs {
  int E = 0;
  const double *U = nullptr;      // [nS][E][nF]
  const double *dUc = nullptr;    // [nFp][E][nF] LDG jumps
  const double *JGinv = nullptr;
  const double *detJ = nullptr;
  double *dUs = nullptr;          // [nDims][nS][E][nF]
  double *dUf = nullptr;          // [nDims][nFp][E][nF]
  long long sStride = 0, fStride = 0;
};
void launch_faces_ldg(int nDims, const FaceTable &ft, const double *Ufpts, double *dUc, const Phys &ph,
                      cudaStream_t st);
void launch_elem_grad(int nDims, int order, const GradArgs &g, const TpTables &t, cudaStream_t st);
void launch_faces_visc(int nDims, const FaceTable &ft, const double *Ufpts, const double *dUf, long long fStride,
                       double *Fn, double *waveSp, const Phys &ph, cudaStream_t st);
// tensor-product element stage with the viscous flux added at the solution points
void launch_element_stage_tp_visc(int nDims, int order, const ElemArgs &a, const TpTables &t, cudaStream_t st);

// Wave speed at every flux point from U_fpts (reference: ele.cpp:1076-1125).
void launch_wavesp_init(int nDims, int nFp, int E, const double *Ufpts, const double *norm,
                        double gamma, double *waveSp, cudaStream_t st);

// Element CFL time step (reference: ele.cpp:1127-1146) and its minimum.
void launch_element_dt(int nDims, int nS, int nFp, int nPF, int E, const double *detJ,
                       const double *wSpt, const double *wSurf, const double *waveSp,
                       const double *dA, double cflFac, double *eleDt,
                       unsigned long long *dtMinBits, cudaStream_t st);
void launch_reset_min(unsigned long long *bits, cudaStream_t st);
void launch_store_min(const unsigned long long *bits, double *dt, double *time_acc,
                      cudaStream_t st);
void launch_add_time(const double *dt, double *time_acc, cudaStream_t st);

// out[i] = x[i] + sgn * y[i] (sgn = +1 or -1), the elementwise updates of the
// P-multigrid cycle (reference: multigrid.cpp:199-205, 282-290, 366-384).
void launch_add(long long n, double *out, const double *x, const double *y, double sgn, cudaStream_t st);

// Per-element residual norm contributions (reference: ele.cpp:1922-1944).
void launch_residual_norm(int nS, int E, int nF, const double *divF, const double *detJ,
                          const double *wSpt, int resType, double *eleRes, cudaStream_t st);

// Device health: counts non-finite or non-positive density entries in U.
void launch_check_state(int nS, int E, int nF, const double *U, unsigned int *bad,
                        cudaStream_t st);

}  // namespace frk
