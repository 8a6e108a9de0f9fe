// Launch interface of the per-stage FR kernels.
// All arrays are device pointers in the reference layout
// ([point][element][field], last index fastest).  Kernels are templated on
// the working type R: double for the plain form, float for the precision
// form (FP32 state, fluxes and operator tables; time step, metrics at setup
// and the norm reductions stay FP64).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <vector>

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

// The same for data of the working type R (the precision form's state).
template <typename R>
void launch_apply_op_t(const Csr &A, const R *in, R *out, long long N, cudaStream_t st);

// Face-point table, one entry per flux point of each face, sorted by left slot.
template <typename R>
struct FaceTableT {
  int n = 0;
  int nInterior = 0;            // interior points first, then boundary points
  const int *slotL = nullptr;   // fpt*E + e of the left side
  const int *slotR = nullptr;   // fpt*E + e of the right side, or -(bc+2) on a boundary
  const R *nrm = nullptr;       // [n][nDims] left unit normal
  const R *dAL = nullptr;
  const R *dAR = nullptr;
};
using FaceTable = FaceTableT<double>;

// Common inviscid flux on every face point: Fn_fpts at both sides and the
// left-side wave speed (reference: solver.cpp:752-758, face.cpp:163-208).
// Interior and boundary points run as two kernels (no BC code in the
// interior one).  The wave speed is kept in FP64 for the time step.
template <typename R>
void launch_faces_inviscid(int nDims, const FaceTableT<R> &ft, const R *Ufpts, R *Fn, double *waveSp,
                           const Phys &ph, cudaStream_t st);

// One part of a case split by a partition of its elements (emulated ranks on
// one device, or one rank): the face points the partition cuts, each formed
// with this part's element as the left side and the peer's trace, received
// for every stage, as the right state (mpiFace::getRightState,
// src/mpiFace.cpp:158-175).  Points are listed by peer part, and per peer in
// the order both sides share (by face, then by the face's left point order),
// so the k-th trace one side sends is the k-th the other receives.
constexpr int kMaxParts = 64;
template <typename R>
struct CutTableT {
  int n = 0;
  const int *slot = nullptr;  // fpt*E + e of this part's side
  const int *left = nullptr;  // 1 where this side is the face's left side in the unsplit mesh
  const R *nrm = nullptr;     // [n][nDims] this side's unit normal
  const R *dA = nullptr;      // [n] this side's dA
  R *send = nullptr;          // [n][nF] this side's traces, packed for every stage
  R *recv = nullptr;          // [n][nF] the peers' traces at the same points
};

// send[i] = U_fpts at slot[i], all fields.
template <typename R>
void launch_pack_cut(int nF, const CutTableT<R> &c, const R *Ufpts, cudaStream_t st);
// Common flux at the cut points from this side's trace and recv (Rusanov,
// or 2-D Roe), written to this side's Fn; wave speed where `left`.
template <typename R>
void launch_faces_cut(int nDims, const CutTableT<R> &c, const R *Ufpts, R *Fn, double *waveSp, const Phys &ph,
                      cudaStream_t st);
// dts[0..n) (device scalars, n <= kMaxParts) all set to their minimum.
void launch_min_dt(double *const *dts, int n, cudaStream_t st);

enum ElemMode : int {
  MODE_RESIDUAL = 0,  // calcResidual only: divF -> divF_out
  MODE_RK_STAGE = 1,  // standard RK intermediate stage (timeStepA + running timeStepB)
  MODE_RK_FINAL = 2,  // standard RK final stage (remaining timeStepB)
  MODE_JAMESON = 3    // Jameson-form stage: U = U0 - RKa[s+1] divF/detJ dt
};

// RK update of one stage.  Plain form (double): `acc` is the running
// final-stage sum U0 - sum_j RKb_j dt divF_j/detJ, as timeStepB forms it.
// Precision form (float): `acc` holds only the increments
// -sum_j RKb_j dt divF_j/detJ, and the state is the pair (U, comp) with U the
// float nearest the FP64 value and comp the rounding remainder; the final
// stage adds the increments to that pair by an error-free (TwoSum) addition,
// so the step-to-step accumulation keeps ~48 bits although every array is
// FP32 (Kahan-compensated RK sums).
template <typename R>
struct ElemArgsT {
  int E = 0, nS = 0, nFp = 0, EB = 1;
  const R *U = nullptr;            // current stage state [nS][E][nF]
  const R *JGinv = nullptr;        // [nDims][nS][E][nDims]
  const R *detJ = nullptr;         // [nS][E]
  const R *Fn = nullptr;           // common normal flux * dA [nFp][E][nF]
  Csr grad[3], extFn[3], corr, ext;
  int mode = MODE_RESIDUAL;
  int stage = 0;
  int nRK = 4;
  double rka_next = 0.0, rkb = 0.0;
  const double *dt = nullptr;      // device scalar
  const double *eleDt = nullptr;   // per-element dt (dtType 2) or null
  const R *src = nullptr;          // P-multigrid source or null
  R *U0 = nullptr;                 // RK base state (written at stage 0)
  R *acc = nullptr;                // running final-stage sum (see above)
  R *comp = nullptr;               // precision form: rounding remainder of U
  R *Uout = nullptr;               // next state
  R *divF_out = nullptr;           // optional divF of this stage
  R *Ufpts_out = nullptr;          // optional: next state at flux points
  R *F_dbg = nullptr;              // optional: F_spts [nDims][nS][E][nF]
  R *disFn_dbg = nullptr;          // optional: Fn - extrapolated flux [nFp][E][nF]
  unsigned int *err = nullptr;     // device status word (bit 0: a bounded wait ran out)
  double gamma = 1.4;
  // viscous stages: physical gradient at the solution points
  // [nDims][nS][E][nF] (stride between dimensions dUsStride), and constants
  const R *dUs = nullptr;
  long long dUsStride = 0;
  Phys ph{};
};
using ElemArgs = ElemArgsT<double>;

size_t elem_smem_bytes(int nDims, int nS, int nFp, int EB);
void launch_element_stage(int nDims, const ElemArgs &a, cudaStream_t st);

// Tensor-product form of the same operators (quads/hexes): the dense
// matrices' nonzeros, verified bitwise on the host, as 1-D tables.
//   grad_d[s][c] = D[i_d(s)][m]   for c on the line through s along d
//   ext[f][s]    = E1[side(f)][m] for s on the line of f (normal dim dn(f))
//   extFn_dn     = (side ? +1 : -1) * ext
//   corr[s][f]   = corrVal[s][face] at f = corrFpt[s][face], one per face
template <typename R>
struct TpTablesT {
  const R *D = nullptr;             // [n][n]
  const R *E1 = nullptr;            // [2][n]   side 0: xi=-1, side 1: xi=+1
  const R *EFn1 = nullptr;          // [2][n]   E1 times the reference normal
  const int *fptBase = nullptr;     // [nFp] first solution point of the line
  const int *fptDn = nullptr;       // [nFp] normal dimension
  const int *fptSide = nullptr;     // [nFp]
  const int *linePair = nullptr;    // [nFp/2] the two ends of a line: side-0 fpt | side-1 fpt << 16
  const int *corrFpt = nullptr;     // [nS][2*nDims]
  const R *corrVal = nullptr;       // [nS][2*nDims]
  const R *lineCorr = nullptr;      // [2][n] corrVal by side and index along the face normal
};
using TpTables = TpTablesT<double>;
bool tp_supported(int nDims, int order);

// Many cases of uneven order advanced by one element launch per RK stage
// (the batch's many-order form): a persistent kernel whose CTAs take element
// blocks of every order group from a device work counter and run the
// tensor-product stage of that group's order on each (CTAs have the threads
// and shared memory of the largest block).  The last CTA to finish resets the
// counters and, on the last stage of a step, advances every group's time.
constexpr int kMaxOrderGroups = 6;
template <typename R>
struct MultiElemArgsT {
  int nGroups = 0;
  int total = 0;                         // element blocks over all groups
  int order[kMaxOrderGroups] = {};
  int start[kMaxOrderGroups + 1] = {};   // first work item of each group
  ElemArgsT<R> a[kMaxOrderGroups];
  TpTablesT<R> t[kMaxOrderGroups];
  unsigned int *next = nullptr, *done = nullptr;  // zero between launches
  double *timeAcc[kMaxOrderGroups] = {};          // final stage: timeAcc += *dt per group
  int finalStage = 0;
};
// The face points of all groups in one launch: interior points of group g
// are work items istart[g] .. istart[g+1]-1, its boundary points follow all
// interior ones at bstart[g].
template <typename R>
struct MultiFaceArgsT {
  int nGroups = 0;
  int istart[kMaxOrderGroups + 1] = {}, bstart[kMaxOrderGroups + 1] = {};
  FaceTableT<R> ft[kMaxOrderGroups];
  const R *Uf[kMaxOrderGroups] = {};
  R *Fn[kMaxOrderGroups] = {};
  double *wave[kMaxOrderGroups] = {};
};
template <typename R>
void launch_element_stage_multi(int nDims, const MultiElemArgsT<R> &m, cudaStream_t st);
template <typename R>
void launch_faces_multi(int nDims, const MultiFaceArgsT<R> &m, const Phys &ph, cudaStream_t st);


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
  CUtensorMap comp;   // [nS][E*nF]    precision form: rounding remainder of U
  // viscous stages
  CUtensorMap dUs;    // [nDims][nS][E*nF]   physical gradient at the solution points
  CUtensorMap dUc;    // [nFp][E*nF]         LDG jumps
  CUtensorMap dUf;    // [nDims][nFp][E*nF]  gradient at the flux points
};
// Elements per CTA of the TMA kernel for (nDims, order, working type); the
// precision form has several instantiations (tile shapes) and `variant`
// picks one of them (0 .. tma_variants()-1), chosen by the autotuner.
int tma_variants(bool fp32);
template <typename R>
int tma_elems_per_block(int nDims, int order, int variant = 0);
template <typename R>
size_t tma_smem_bytes(int nDims, int order, int variant = 0);
template <typename R>
void launch_element_stage_tma(int nDims, int order, const ElemArgsT<R> &a, const TpTablesT<R> &t,
                              const TmaMaps &m, cudaStream_t st, int variant = 0);
// The same with the viscous flux added at the solution points; the gradient
// tiles (TmaMaps::dUs) arrive by TMA.  Tile variant 0.
template <typename R>
void launch_element_stage_tma_visc(int nDims, int order, const ElemArgsT<R> &a, const TpTablesT<R> &t,
                                   const TmaMaps &m, cudaStream_t st);
// Corrected physical gradient at the solution and flux points with TMA tiles
// (U, dUc, JGinv, detJ in; dUs, dUf out), element block of tile variant 0.
template <typename R>
void launch_elem_grad_tma(int nDims, int order, int E, const TpTablesT<R> &t, const TmaMaps &m,
                          unsigned int *err, cudaStream_t st);
// Precision-form element stage on the tensor cores (tcgen05 kind::tf32,
// 3xTF32) for 2-D orders 1..4 (32 elements per CTA) and 3-D order 1 (24);
// the tile variant after the CUDA-core ones.  The operators are packed once
// on the host into the MMA operand layout (grad/extFn: nDims pointers).
bool tc_supported(int nDims, int order);
int tc_elems_per_block(int nDims, int order);
bool tc_pack_ops(int nDims, int order, const double *const grad[3], const double *const extFn[3],
                 const double *corr, const double *ext, std::vector<float> &blob);
size_t tc_smem_bytes(int nDims, int order);
void launch_element_stage_tc(int nDims, int order, const ElemArgsT<float> &a, const float *ops, const TmaMaps &m,
                             cudaStream_t st);
template <typename R>
int tp_elems_per_block(int nDims, int order);
template <typename R>
void launch_element_stage_tp(int nDims, int order, const ElemArgsT<R> &a, const TpTablesT<R> &t,
                             cudaStream_t st);

// Viscous (LDG) stage pieces (kernels/stage_visc.cu).
template <typename R>
struct GradArgsT {
  int E = 0;
  const R *U = nullptr;      // [nS][E][nF]
  const R *dUc = nullptr;    // [nFp][E][nF] LDG jumps
  const R *JGinv = nullptr;
  const R *detJ = nullptr;
  R *dUs = nullptr;          // [nDims][nS][E][nF]
  R *dUf = nullptr;          // [nDims][nFp][E][nF]
  long long sStride = 0, fStride = 0;
};
using GradArgs = GradArgsT<double>;
template <typename R>
void launch_faces_ldg(int nDims, const FaceTableT<R> &ft, const R *Ufpts, R *dUc, const Phys &ph,
                      cudaStream_t st);
template <typename R>
void launch_elem_grad(int nDims, int order, const GradArgsT<R> &g, const TpTablesT<R> &t, cudaStream_t st);
template <typename R>
void launch_faces_visc(int nDims, const FaceTableT<R> &ft, const R *Ufpts, const R *dUf, long long fStride,
                       R *Fn, double *waveSp, const Phys &ph, cudaStream_t st);
// tensor-product element stage with the viscous flux added at the solution points
template <typename R>
void launch_element_stage_tp_visc(int nDims, int order, const ElemArgsT<R> &a, const TpTablesT<R> &t,
                                  cudaStream_t st);

// Wave speed at every flux point from U_fpts (reference: ele.cpp:1076-1125).
template <typename R>
void launch_wavesp_init(int nDims, int nFp, int E, const R *Ufpts, const double *norm, double gamma,
                        double *waveSp, cudaStream_t st);

// Element CFL time step (reference: ele.cpp:1127-1146) and its minimum.
void launch_element_dt(int nDims, int nS, int nFp, int nPF, int E, const double *detJ,
                       const double *wSpt, const double *wSurf, const double *waveSp,
                       const double *dA, double cflFac, double *eleDt,
                       unsigned long long *dtMinBits, cudaStream_t st);
// The same, the minimum stored straight into *dt by the last block, which
// then resets *bits (to +inf) and *count (to 0): one launch per time step.
void launch_element_dt_min(int nS, int nFp, int nPF, int E, const double *detJ, const double *wSpt,
                           const double *wSurf, const double *waveSp, const double *dA, double cflFac, double *eleDt,
                           unsigned long long *bits, unsigned int *count, double *dt, cudaStream_t st);
void launch_reset_min(unsigned long long *bits, cudaStream_t st);
void launch_store_min(const unsigned long long *bits, double *dt, double *time_acc,
                      cudaStream_t st);
void launch_add_time(const double *dt, double *time_acc, cudaStream_t st);

// out[i] = x[i] + sgn * y[i] (sgn = +1 or -1), the elementwise updates of the
// P-multigrid cycle (reference: multigrid.cpp:199-205, 282-290, 366-384).
void launch_add(long long n, double *out, const double *x, const double *y, double sgn, cudaStream_t st);
void launch_add32(long long n, float *out, const float *x, const float *y, double sgn, cudaStream_t st);

// Per-element residual norm contributions (reference: ele.cpp:1922-1944),
// accumulated in FP64 whatever the type of divF.
template <typename R>
void launch_residual_norm(int nS, int E, int nF, const R *divF, const double *detJ,
                          const double *wSpt, int resType, double *eleRes, cudaStream_t st);

// Device health: counts non-finite or non-positive density entries in U.
template <typename R>
void launch_check_state(int nS, int E, int nF, const R *U, unsigned int *bad, cudaStream_t st);

// Precision-form conversions at the boundary and at setup:
//   split   : U64 -> (U32 = fl32(U64), comp = fl32(U64 - U32))
//   join    : (U32, comp) -> U64 = U32 + comp
//   narrow  : FP64 -> FP32 (metrics, normals, face areas)
//   widen   : FP32 -> FP64 (residuals, traces read back by tools)
// ---- moving meshes (motion.cu), FP64 ------------------------------------
struct MotionArgs {
  int type = 0, nDims = 2, nVerts = 0, E = 0, nS = 0, nFp = 0, nNodes = 0;
  const double *time = nullptr, *dt = nullptr;  // device scalars
  double DX = 0, DY = 0, Ax = 0, Ay = 0, Fx = 0, Fy = 0, Ar = 0, Fr = 0;
  const double *xv0 = nullptr, *rv0 = nullptr;  // initial vertices [nVerts][nDims], (r, theta, psi)
  double *xv = nullptr, *gv = nullptr;          // moved vertices and their velocities
  const int *c2v = nullptr;                     // [E][nNodes]
  const double *shape = nullptr, *dshape = nullptr;  // [nS + nFp][nNodes] and [..][nNodes][nDims]
  const double *tNorm = nullptr;                // [nFp][nDims]
  double *Jac = nullptr;                        // [nDims][nS][E][nDims], d x_comp / d xi_dim
  double *JGinv = nullptr, *detJ = nullptr, *norm = nullptr, *dA = nullptr;
  double *gVs = nullptr, *gVf = nullptr;        // grid velocity [nS|nFp][E][nDims]
  const double *opGrad = nullptr;               // [nDims][nS][nS] dense
  const double *opExt = nullptr;                // [nFp][nS]
  const double *opCorr = nullptr;               // [nS][nFp]
  unsigned int *err = nullptr;                  // bit 2: negative Jacobian
};
struct MotionStages {
  const double *divF[8];
  double rkb[8];
  int n = 0;
};
void launch_move_vertices(const MotionArgs &m, double rkVal, cudaStream_t st);
void launch_motion_geometry(const MotionArgs &m, bool transforms, cudaStream_t st);
void launch_face_refresh(const FaceTableT<double> &ft, int nDims, const double *norm, const double *dA,
                         cudaStream_t st);
void launch_faces_motion(int nDims, const FaceTableT<double> &ft, const double *Uf, double *Fn, double *waveSp,
                         const double *gVf, const Phys &ph, cudaStream_t st);
void launch_wavesp_motion(int nDims, int nFp, int E, const double *Uf, const double *norm, const double *gVf,
                          double gamma, double *waveSp, cudaStream_t st);
void launch_motion_residual(const MotionArgs &m, const double *U, const double *Fn, double gamma, double *F,
                            double *disFn, double *divF, cudaStream_t st);
// src: the P-multigrid source term added to every stage residual, or null
void launch_motion_step_a(long long nSE, int nF, int E, const double *U0, const double *divF, const double *src,
                          const double *detJ, const double *dt, const double *eleDt, double rk, double *U,
                          cudaStream_t st);
void launch_motion_step_b(long long nSE, int nF, int E, const double *base, const MotionStages &stages,
                          const double *src, const double *detJ, const double *dt, const double *eleDt, double *U,
                          cudaStream_t st);

// ---- boundary monitors: wall forces and mass flux (monitor.cu) -----------
template <typename R>
struct MonitorArgsT {
  int E = 0, nPF = 0, nI = 0, n = 0;       // face-point table: boundary points are [nI, n)
  const int *slotL = nullptr, *slotR = nullptr;
  const R *nrm = nullptr, *dAL = nullptr;
  const R *Uf = nullptr, *Fn = nullptr;    // U_fpts, Fn_fpts (= common flux * dA)
  const R *dUf = nullptr;                  // viscous: gradient at the flux points, else null
  long long fStride = 0;                   // dUf stride between dimensions
  const double *wSurf = nullptr;           // [nPF] Gauss weights within a face
  Phys ph{};
  int errorNorm = 0;
  double *part = nullptr;                  // [n - nI][11] scratch
};
// out[0..5]: pressure and viscous force (x, y, z each); out[6..]: mass flux per field.
template <typename R>
void launch_boundary_monitors(int nDims, const MonitorArgsT<R> &a, double *out, cudaStream_t st);

// ---- error integrals against the exact solution (error.cu) ---------------
struct ErrorArgs {
  int nDims = 2, nS = 0, nQ = 0, E = 0, nF = 0, nNodes = 0;
  int icType = 0, testCase = 0, errorNorm = 0;
  double gamma = 1.4, pIC = 1, rhoIC = 1, vortexAngle = 0, pi = 0;
  double xmin = -5, xmax = 5, ymin = -5, ymax = 5;  // periodic box of the exact vortex
  const double *time = nullptr;                     // device scalar
  const double *U = nullptr, *detJ = nullptr;       // [nS][E][nF], [nS][E]
  const double *opQ = nullptr, *wQ = nullptr;       // [nQ][nS] spts -> evaluation points, weights
  const double *shapeQ = nullptr;                   // [nQ][nNodes]
  const double *xv = nullptr;                       // vertex positions [nVerts][nDims]
  const int *c2v = nullptr;                         // [E][nNodes]
  double *elemErr = nullptr, *elemU = nullptr;      // per-element integrals [E][nF]
};
void launch_error_integral(const ErrorArgs &a, double *out, cudaStream_t st);

// Primitive variables at the plot points from the FP64 state (output only).
void launch_plot_primitives(int nDims, const double *U, const double *opp, double *Vp, int nS, int nP, int E,
                            double gamma, cudaStream_t st);
void launch_split(long long n, const double *U64, float *U32, float *comp, cudaStream_t st);
void launch_join(long long n, const float *U32, const float *comp, double *U64, cudaStream_t st);
void launch_narrow(long long n, const double *in, float *out, cudaStream_t st);
void launch_widen(long long n, const float *in, double *out, cudaStream_t st);

}  // namespace frk
