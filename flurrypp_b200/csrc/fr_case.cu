// fr_case: one FR solver instance on the GPU, and the C ABI (include/fr_b200.h).
//
// The host side mirrors the reference `solver` (src/solver.cpp): setup builds
// mesh, faces, operators and metrics on the host, then everything the stages
// touch lives in device memory for the life of the case.  update() issues the
// same sequence of steps as solver::update (solver.cpp:319-363), each stage as
// a face kernel plus a fused element kernel.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <type_traits>
#include <vector>

#include <dlfcn.h>
#include <nccl.h>

#include "../../include/fr_b200.h"
#include "host/fr_host.hpp"
#include "kernels/launch.cuh"
#include "kernels/stage.hpp"

namespace {

struct DevBuf {
  void *p = nullptr;
  size_t bytes = 0;
  bool fp32 = false;
};

// FP32 device arrays of the live cases, begin -> end address: the
// no-allocation norm takes raw FP64 pointers and refuses these
std::mutex g_fp32Mu;
std::map<uintptr_t, uintptr_t> g_fp32Arrays;

void note_fp32(void *p, size_t bytes, bool add) {
  std::lock_guard<std::mutex> lk(g_fp32Mu);
  if (add)
    g_fp32Arrays[(uintptr_t)p] = (uintptr_t)p + bytes;
  else
    g_fp32Arrays.erase((uintptr_t)p);
}

}  // namespace

bool fr_internal_is_fp32(const void *p) {
  const uintptr_t a = (uintptr_t)p;
  std::lock_guard<std::mutex> lk(g_fp32Mu);
  auto it = g_fp32Arrays.upper_bound(a);
  if (it == g_fp32Arrays.begin()) return false;
  --it;
  return a >= it->first && a < it->second;
}

// NCCL, resolved at run time from the libnccl.so.2 the process already has
// (a torch process loads its own) or the system's, so that the library never
// brings a second NCCL into a process.  Used only by parts of a case split
// across ranks (fr_part_create).
struct NcclApi {
  bool ok = false;
  decltype(&ncclSend) send = nullptr;
  decltype(&ncclRecv) recv = nullptr;
  decltype(&ncclGroupStart) groupStart = nullptr;
  decltype(&ncclGroupEnd) groupEnd = nullptr;
  decltype(&ncclAllReduce) allReduce = nullptr;
  decltype(&ncclGetUniqueId) uniqueId = nullptr;
  decltype(&ncclCommInitRank) initRank = nullptr;
  decltype(&ncclCommDestroy) destroy = nullptr;
};
static const NcclApi &nccl_api() {
  static NcclApi api = [] {
    NcclApi a;
    void *h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_NOLOAD);
    if (!h) h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
    if (!h) return a;
    a.send = (decltype(a.send))dlsym(h, "ncclSend");
    a.recv = (decltype(a.recv))dlsym(h, "ncclRecv");
    a.groupStart = (decltype(a.groupStart))dlsym(h, "ncclGroupStart");
    a.groupEnd = (decltype(a.groupEnd))dlsym(h, "ncclGroupEnd");
    a.allReduce = (decltype(a.allReduce))dlsym(h, "ncclAllReduce");
    a.uniqueId = (decltype(a.uniqueId))dlsym(h, "ncclGetUniqueId");
    a.initRank = (decltype(a.initRank))dlsym(h, "ncclCommInitRank");
    a.destroy = (decltype(a.destroy))dlsym(h, "ncclCommDestroy");
    a.ok = a.send && a.recv && a.groupStart && a.groupEnd && a.allReduce && a.uniqueId && a.initRank && a.destroy;
    return a;
  }();
  return api;
}

// cases with fewer solution points than this do not time tile variants
constexpr long long kTuneMinPoints = 1LL << 18;

struct fr_case {
  std::string err;
  fr_setup_opts opts;
  fr::Input in;
  fr::Mesh mesh;
  fr::Geometry geo;
  fr::Operators op;
  std::vector<fr::Face> faces;
  int nDims = 0, nF = 0, nS = 0, nFp = 0, E = 0, nPF = 0, nRK = 0;
  long long iter = 0;
  long long launches = 0;  // kernels launched (graph replays counted per kernel)
  int graphKernels = 0;    // kernels in the captured step
  double hostDt = 0.0;
  bool stateSet = false;
  bool fptsFresh = false;  // U_fpts holds the extrapolation of U_spts
  cudaStream_t stream = nullptr;
  std::vector<DevBuf> allocs;

  // device arrays
  double *U = nullptr, *U0 = nullptr, *acc = nullptr, *Ufpts = nullptr, *Fn = nullptr;
  std::vector<double *> divF;
  double *waveSp = nullptr, *detJ = nullptr, *JGinv = nullptr, *norm = nullptr, *dA = nullptr;
  double *wSpt = nullptr, *wSurf = nullptr, *eleDt = nullptr, *dt = nullptr, *timeAcc = nullptr;
  double *eleRes = nullptr, *src = nullptr;
  double *Fdbg = nullptr, *disFnDbg = nullptr;
  double *dUc = nullptr, *dUs = nullptr, *dUf = nullptr;  // viscous: LDG jumps, gradients
  unsigned long long *dtBits = nullptr;
  unsigned int *dtCount = nullptr;  // blocks done in the fused dt kernel
  unsigned int *bad = nullptr;
  frk::FaceTable ft;
  frk::Csr grad[3], extFn[3], corr, ext;
  frk::TpTables tp;
  bool useTp = false;
  frk::TmaMaps tm;
  bool useTma = false;
  unsigned int *devErr = nullptr;
  int EB = 1;
  frk::Phys ph{};
  cudaGraphExec_t graph = nullptr;
  // kRunChunk steps in one graph, for runs of at least that many steps (one
  // graph launch instead of kRunChunk)
  static constexpr int kRunChunk = 10;
  cudaGraphExec_t graphK = nullptr;
  int graphKernelsK = 0;
  bool ownStream = false;
  bool hostOnly = false;  // set up without a device: setup arrays only
  // P-multigrid (reference: multigrid.cpp:47-384): coarse levels share the
  // mesh and the stream; index = order, null below lowOrder
  std::vector<std::unique_ptr<fr_case>> levels;
  bool pmgCoarse = false;
  // batch group: several cases merged along the element axis, each with its
  // own fixed dt held per element
  bool perElementDt = false;
  double *sol = nullptr, *corrPmg = nullptr;
  float *src32 = nullptr;  // precision form: the P-multigrid source in FP32
  frk::Csr restrictOp, prolongOp;
  // precision form (FR_PREC_MIXED): the stage arrays in FP32; U (FP64) is
  // the boundary copy, and detJ, norm, dA, waveSp, the time step and the
  // norm reductions stay FP64
  bool mixed = false;
  // programmatic dependent launch for cases whose grids fit in about one wave
  // (a solution point per thread: 148 SMs x 1024 threads)
  bool usePdl = false;
  int variant64 = 0;              // plain form: element tile variant in use
  std::vector<float> tuneMs64;    // plain form: element-stage ms per tile variant
  struct Fp32 {
    float *U = nullptr, *U0 = nullptr, *acc = nullptr, *comp = nullptr, *Ufpts = nullptr, *Fn = nullptr;
    float *JGinv = nullptr, *detJ = nullptr;
    std::vector<float *> divF;
    float *dUc = nullptr, *dUs = nullptr, *dUf = nullptr, *Fdbg = nullptr, *disFnDbg = nullptr;
    frk::FaceTableT<float> ft;
    frk::TpTablesT<float> tp;
    frk::TmaMaps tm;
    bool useTma = false;
    int variant = 0;
    float *tcOps = nullptr;     // 2-D tensor-core variant: operators in MMA layout
    std::vector<float> tuneMs;  // element-stage time per tile variant (autotuner)
  } f32;

  // moving mesh (deck "motion" 1..5): the vertex law, the metrics rebuilt at
  // every RK stage and the chain-rule residual (kernels/motion.cu)
  struct MotionState {
    bool on = false;
    frk::MotionArgs a;
    double *F = nullptr, *disFn = nullptr;  // physical flux at spts; Fn - extrapolated normal flux
    unsigned int *err = nullptr;
  } mo;

  // error integrals (testCase 1): evaluation tables for the solution-point
  // (errorNorm 0) and Gauss-Legendre (1, 2) quadratures, built on first use
  struct ErrorTables {
    int nQ = 0;
    double *opQ = nullptr, *wQ = nullptr, *shapeQ = nullptr;
  } errT[2];
  double *errXv = nullptr, *errElem = nullptr, *errOut = nullptr;
  double *monPart = nullptr, *monOut = nullptr;  // boundary monitors: per-point parts, totals

  // one part of a case split by a partition (fr_shard_*): the face points
  // the partition cuts; their right traces arrive in cut.recv before every
  // face pass (the shard packs and exchanges them for all parts)
  frk::CutTableT<double> cut;
  std::vector<int> cutPeer;  // peer part of every cut point (sorted by peer)
  // a part on its own rank (fr_part_create): the traces travel by NCCL
  // send/receive pairs on the case's stream at every face pass, and dt is
  // the NCCL minimum over the ranks; the in-process shard leaves this null
  // and exchanges itself
  ncclComm_t comm = nullptr;
  std::vector<int> segPeer;
  std::vector<long long> segOff, segCount;
  bool ncclOk = true;
  void exchange_nccl() {
    const NcclApi &api = nccl_api();
    frk::launch_pack_cut<double>(nF, cut, Ufpts, stream);
    launches++;
    api.groupStart();
    for (size_t i = 0; i < segPeer.size(); i++) {
      const size_t n = (size_t)segCount[i] * nF;
      if (api.send(cut.send + segOff[i] * nF, n, ncclDouble, segPeer[i], comm, stream) != ncclSuccess ||
          api.recv(cut.recv + segOff[i] * nF, n, ncclDouble, segPeer[i], comm, stream) != ncclSuccess)
        ncclOk = false;
    }
    if (api.groupEnd() != ncclSuccess) ncclOk = false;
  }

  // wall forces and mass flux from the face data of the last residual
  // evaluation (boundFace::computeWallForce / computeMassFlux)
  bool boundary_monitors(int errorNorm, double *host11) {
    const int nB = ft.n - ft.nInterior;
    if (!monOut && (!alloc(monPart, (size_t)std::max(nB, 1) * 11) || !alloc(monOut, 11))) return false;
    if (!mixed) {
      frk::MonitorArgsT<double> a;
      a.E = E, a.nPF = nPF, a.nI = ft.nInterior, a.n = ft.n;
      a.slotL = ft.slotL, a.slotR = ft.slotR, a.nrm = ft.nrm, a.dAL = ft.dAL;
      a.Uf = Ufpts, a.Fn = Fn, a.dUf = in.viscous ? dUf : nullptr, a.fStride = (long long)nFp * E * nF;
      a.wSurf = wSurf, a.ph = ph, a.errorNorm = errorNorm, a.part = monPart;
      frk::launch_boundary_monitors<double>(nDims, a, monOut, stream);
    } else {
      frk::MonitorArgsT<float> a;
      a.E = E, a.nPF = nPF, a.nI = f32.ft.nInterior, a.n = f32.ft.n;
      a.slotL = f32.ft.slotL, a.slotR = f32.ft.slotR, a.nrm = f32.ft.nrm, a.dAL = f32.ft.dAL;
      a.Uf = f32.Ufpts, a.Fn = f32.Fn, a.dUf = in.viscous ? f32.dUf : nullptr, a.fStride = (long long)nFp * E * nF;
      a.wSurf = wSurf, a.ph = ph, a.errorNorm = errorNorm, a.part = monPart;
      frk::launch_boundary_monitors<float>(nDims, a, monOut, stream);
    }
    launches += 2;
    if (cudaMemcpyAsync(host11, monOut, 11 * sizeof(double), cudaMemcpyDeviceToHost, stream) != cudaSuccess)
      return fail(FR_ERR_CUDA, "cudaMemcpy D2H failed");
    return sync();
  }
  int *errC2v = nullptr;

  // solution output: primitive variables at the plot points, copied to a
  // pinned host buffer on a side stream so that stepping goes on meanwhile
  struct Checkpoint {
    double *opp = nullptr;   // [nPpts][nSpts] spts -> plot points
    double *Vp = nullptr;    // [nPpts][E][nF], then the time
    double *host = nullptr;  // pinned copy of Vp
    double *xv = nullptr, *xvHost = nullptr;  // moving mesh: vertex positions, then velocities, at the snapshot
    std::vector<double> gridVel;              // moving mesh: grid velocity at the plot points
    cudaStream_t copy = nullptr;
    cudaEvent_t ready = nullptr, done = nullptr;
    bool pending = false;
    long long iter = 0;
    int nP = 0;
    std::vector<double> pos;  // plot-point positions [nPpts][E][nDims]
  } cp;

  ~fr_case() {
    if (cp.copy) cudaStreamSynchronize(cp.copy);
    if (cp.host) cudaFreeHost(cp.host);
    if (cp.xvHost) cudaFreeHost(cp.xvHost);
    if (cp.ready) cudaEventDestroy(cp.ready);
    if (cp.done) cudaEventDestroy(cp.done);
    if (cp.copy) cudaStreamDestroy(cp.copy);
    if (stream) cudaStreamSynchronize(stream);
    if (graph) cudaGraphExecDestroy(graph);
    if (graphK) cudaGraphExecDestroy(graphK);
    levels.clear();  // coarse levels use this case's stream: release them first
    for (auto &b : allocs) {
      if (b.fp32) note_fp32(b.p, b.bytes, false);
      cudaFree(b.p);
    }
    if (ownStream && ownedStream) cudaStreamDestroy(ownedStream);
  }
  cudaStream_t ownedStream = nullptr;

  int errCode = 0;  // the FR_ERR_* of the last fail()
  bool fail(int code, const std::string &m) {
    err = m;
    errCode = code;
    return false;
  }
  template <typename T>
  bool alloc(T *&p, size_t count) {
    void *q = nullptr;
    size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
    cudaError_t e = cudaMalloc(&q, bytes);
    if (e != cudaSuccess) {
      err = std::string("cudaMalloc: ") + cudaGetErrorString(e);
      errCode = FR_ERR_CUDA;
      return false;
    }
    cudaMemsetAsync(q, 0, bytes, stream);
    const bool fp32 = std::is_same<T, float>::value;
    if (fp32) note_fp32(q, bytes, true);
    allocs.push_back({q, bytes, fp32});
    p = (T *)q;
    return true;
  }
  template <typename T>
  bool upload(T *&p, const std::vector<T> &h) {
    if (!alloc(p, h.size())) return false;
    cudaError_t e = cudaMemcpyAsync(p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) {
      err = std::string("cudaMemcpy: ") + cudaGetErrorString(e);
      errCode = FR_ERR_CUDA;
      return false;
    }
    return true;
  }
  bool cuda_ok(const char *what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
      err = std::string(what) + ": " + cudaGetErrorString(e);
      return false;
    }
    return true;
  }

  bool make_csr(const std::vector<double> &A, int rows, int cols, frk::Csr &out) {
    std::vector<int> rp(rows + 1, 0), ci;
    std::vector<double> v;
    for (int r = 0; r < rows; r++) {
      for (int c = 0; c < cols; c++) {
        double a = A[(size_t)r * cols + c];
        if (a != 0.0) {
          ci.push_back(c);
          v.push_back(a);
        }
      }
      rp[r + 1] = (int)ci.size();
    }
    int *drp, *dci;
    double *dv;
    if (!upload(drp, rp) || !upload(dci, ci) || !upload(dv, v)) return false;
    out.nRows = rows;
    out.nCols = cols;
    out.rowptr = drp;
    out.col = dci;
    out.val = dv;
    return true;
  }

  bool setup(const fr_setup_opts &o) {
    opts = o;
    hostOnly = o.device < 0;
    if (hostOnly) return setup_host();
    if (cudaSetDevice(o.device) != cudaSuccess) return fail(FR_ERR_CUDA, "cudaSetDevice failed");
    if (!stream) {
      if (cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) != cudaSuccess)
        return fail(FR_ERR_CUDA, "stream create");
      ownStream = true;
      ownedStream = stream;
    }
    if (o.precision != FR_PREC_FP64 && o.precision != FR_PREC_MIXED)
      return fail(FR_ERR_UNSUPPORTED, o.precision == FR_PREC_MIXED_REFINE
                                          ? "FR_PREC_MIXED_REFINE is a form of the solve server"
                                          : "unknown precision");
    mixed = o.precision == FR_PREC_MIXED;
    if (!setup_host()) return false;
    return setup_device();
  }

  // Device buffers, uploads, face table, operator tables (after setup_host or
  // after a merge of several cases' host data).
  bool setup_device() {
    const fr_setup_opts &o = opts;
    size_t nU = (size_t)nS * E * nF, nUf = (size_t)nFp * E * nF;
    if (!alloc(U, nU)) return false;
    if (!mixed) {
      if (!alloc(U0, nU) || !alloc(acc, nU) || !alloc(Ufpts, nUf) || !alloc(Fn, nUf)) return false;
      divF.assign(nRK, nullptr);
      for (int s = 0; s < nRK; s++)
        if (!alloc(divF[s], nU)) return false;
      if (o.debug_arrays)
        if (!alloc(Fdbg, (size_t)nDims * nU) || !alloc(disFnDbg, nUf)) return false;
      if (!upload(JGinv, geo.JGinv_spts)) return false;
    } else {
      if (!alloc(f32.U, nU) || !alloc(f32.U0, nU) || !alloc(f32.acc, nU) || !alloc(f32.comp, nU) ||
          !alloc(f32.Ufpts, nUf) || !alloc(f32.Fn, nUf))
        return false;
      f32.divF.assign(nRK, nullptr);
      for (int s = 0; s < nRK; s++)
        if (!alloc(f32.divF[s], nU)) return false;
      if (o.debug_arrays)
        if (!alloc(f32.Fdbg, (size_t)nDims * nU) || !alloc(f32.disFnDbg, nUf)) return false;
      if (!upload(f32.JGinv, narrow(geo.JGinv_spts)) || !upload(f32.detJ, narrow(geo.detJac_spts))) return false;
    }
    if (!alloc(waveSp, (size_t)nFp * E) || !alloc(eleDt, E) || !alloc(dt, 1) || !alloc(timeAcc, 1) ||
        !alloc(eleRes, (size_t)E * nF) || !alloc(dtBits, 1) || !alloc(dtCount, 1) || !alloc(bad, 1))
      return false;
    frk::launch_reset_min(dtBits, stream);  // the fused dt kernel starts from +inf
    if (!upload(detJ, geo.detJac_spts) || !upload(norm, geo.norm_fpts) || !upload(dA, geo.dA_fpts)) return false;
    if (!upload(wSpt, fr::spt_weights(nDims, in.order)) || !upload(wSurf, fr::face_weights(nDims, in.order)))
      return false;
    for (int d = 0; d < nDims; d++) {
      if (!make_csr(op.grad[d], nS, nS, grad[d])) return false;
      if (!make_csr(op.extFn[d], nFp, nS, extFn[d])) return false;
    }
    if (!make_csr(op.corr, nS, nFp, corr) || !make_csr(op.ext, nFp, nS, ext)) return false;

    // face-point table, sorted by left slot for coalesced gathers
    struct FP {
      int sL, sR;
      double n[3], aL, aR;
    };
    std::vector<FP> fps;
    fps.reserve(faces.size() * nPF);
    for (auto &f : faces)
      for (int j = 0; j < nPF; j++) {
        FP p{};
        int fL = f.locL * nPF + j;
        p.sL = fL * E + f.eL;
        for (int d = 0; d < nDims; d++) p.n[d] = geo.norm_fpts[(size_t)p.sL * nDims + d];
        p.aL = geo.dA_fpts[p.sL];
        if (f.eR >= 0) {
          p.sR = f.fptR[j] * E + f.eR;
          p.aR = geo.dA_fpts[p.sR];
        } else {
          p.sR = -(f.bc + 2);
          p.aR = 0.0;
        }
        fps.push_back(p);
      }
    std::sort(fps.begin(), fps.end(), [](const FP &a, const FP &b) {
      const bool ia = a.sR >= 0, ib = b.sR >= 0;
      if (ia != ib) return ia;  // interior points first
      return a.sL < b.sL;
    });
    int nInt = 0;
    for (auto &p : fps) nInt += p.sR >= 0 ? 1 : 0;
    std::vector<int> sL(fps.size()), sR(fps.size());
    std::vector<double> nrm(fps.size() * nDims), aL(fps.size()), aR(fps.size());
    for (size_t i = 0; i < fps.size(); i++) {
      sL[i] = fps[i].sL;
      sR[i] = fps[i].sR;
      for (int d = 0; d < nDims; d++) nrm[i * nDims + d] = fps[i].n[d];
      aL[i] = fps[i].aL;
      aR[i] = fps[i].aR;
    }
    int *dsL, *dsR;
    if (!upload(dsL, sL) || !upload(dsR, sR)) return false;
    ft.n = f32.ft.n = (int)fps.size();
    ft.nInterior = f32.ft.nInterior = nInt;
    ft.slotL = f32.ft.slotL = dsL;
    ft.slotR = f32.ft.slotR = dsR;
    if (!mixed) {
      double *dn, *daL, *daR;
      if (!upload(dn, nrm) || !upload(daL, aL) || !upload(daR, aR)) return false;
      ft.nrm = dn;
      ft.dAL = daL;
      ft.dAR = daR;
    } else {
      float *dn, *daL, *daR;
      if (!upload(dn, narrow(nrm)) || !upload(daL, narrow(aL)) || !upload(daR, narrow(aR))) return false;
      f32.ft.nrm = dn;
      f32.ft.dAL = daL;
      f32.ft.dAR = daR;
    }

    ph.gamma = in.gamma;
    ph.rhoBound = in.rhoBound;
    ph.uBound = in.uBound;
    ph.vBound = in.vBound;
    ph.wBound = in.wBound;
    ph.pBound = in.pBound;
    ph.TWall = in.TWall;
    ph.RGas = in.RGas;
    ph.uWall = in.uWall;
    ph.vWall = in.vWall;
    ph.wWall = in.wWall;
    ph.mu_inf = in.mu_inf;
    ph.prandtl = in.prandtl;
    ph.rt_inf = in.rt_inf;
    ph.c_sth = in.c_sth;
    ph.penFact = in.penFact;
    ph.tau = in.tau;
    ph.fixVis = in.fixVis;
    ph.viscFluxQuirk = o.visc_flux_quirk;
    ph.riemannType = in.riemannType;

    // elements per block of the fused element kernel
    EB = 1;
    for (int c = 2; c <= 32; c *= 2) {
      if (frk::elem_smem_bytes(nDims, nS, nFp, c) > 72 * 1024) break;
      if ((long long)nS * c > 1024) break;
      EB = c;
    }
    useTp = build_tp() && !opts.generic_kernels;
    if (useTp) EB = mixed ? frk::tp_elems_per_block<float>(nDims, in.order) : frk::tp_elems_per_block<double>(nDims, in.order);
    if (mixed && !useTp) return fail(FR_ERR_UNSUPPORTED, "the precision form needs the tensor-product operators");
    if (in.viscous) {
      if (!useTp) return fail(FR_ERR_UNSUPPORTED, "viscous stages need the tensor-product operators");
      if (!mixed) {
        if (!alloc(dUc, nUf) || !alloc(dUs, (size_t)nDims * nU) || !alloc(dUf, (size_t)nDims * nUf)) return false;
      } else {
        if (!alloc(f32.dUc, nUf) || !alloc(f32.dUs, (size_t)nDims * nU) || !alloc(f32.dUf, (size_t)nDims * nUf))
          return false;
      }
    }
    if (!alloc(devErr, 1)) return false;
    if (in.motion && !setup_motion()) return false;
    usePdl = !opts.no_pdl && (long long)nS * E <= 148LL * 1024;
    if (!mixed) {
      useTma = useTp && !opts.no_tma && build_tma(0);
      if (useTma && in.viscous) EB = frk::tma_elems_per_block<double>(nDims, in.order);
      if (useTma && !in.viscous && !autotune_tiles64()) return false;
    } else if (useTp && in.viscous && !opts.no_tma && (E * nF) % 4 == 0) {
      // viscous precision form: tile variant 0
      if (build_tma32(0)) {
        f32.useTma = true;
        f32.variant = 0;
        EB = frk::tma_elems_per_block<float>(nDims, in.order, 0);
      }
    } else if (useTp && !opts.no_tma && (E * nF) % 4 == 0) {
      if (!autotune_tiles()) return false;
    }
    hostDt = in.dt;
    if (cudaMemcpyAsync(dt, &hostDt, sizeof(double), cudaMemcpyHostToDevice, stream) != cudaSuccess)
      return fail(FR_ERR_CUDA, "dt upload");
    if (in.PMG) {
      if (!alloc(src, nU) || !alloc(sol, nU) || !alloc(corrPmg, nU)) return false;
      if (mixed && !alloc(src32, nU)) return false;
      if (in.order > 0 && !make_csr(op.restrict_, op.nSptsRes, nS, restrictOp)) return false;
      if (!make_csr(op.prolong, op.nSptsPro, nS, prolongOp)) return false;
      if (!pmgCoarse && !build_levels()) return false;
    }
    if (cudaStreamSynchronize(stream) != cudaSuccess) return fail(FR_ERR_CUDA, "setup sync");
    return cuda_ok("setup");
  }

  // Coarse P levels (multiGrid::setup, multigrid.cpp:111-139): each a solver
  // of order P on the same mesh, with the deck's initial condition applied
  // (solver::initializeSolution(true)), which also fixes their initial wave
  // speeds for CFL-based stepping.
  bool build_levels() {
    if (in.lowOrder < 0 || in.lowOrder >= in.order) return in.order == 0 || fail(FR_ERR_ARG, "bad lowOrder");
    levels.clear();
    levels.resize(in.order);
    for (int P = in.lowOrder; P < in.order; P++) {
      std::unique_ptr<fr_case> L(new fr_case());
      L->in = in;
      L->in.order = P;
      L->mesh = mesh;
      L->pmgCoarse = true;
      L->stream = stream;
      if (!L->setup(opts)) return fail(FR_ERR_SETUP, "P-multigrid level " + std::to_string(P) + ": " + L->err);
      std::vector<double> Uic;
      std::string e;
      if (!fr::initial_condition(L->in, L->geo, L->nS, L->E, fr::IC_DECK, nullptr, 0, Uic, e))
        return fail(FR_ERR_SETUP, e);
      if (!L->set_state_host(Uic.data())) return fail(FR_ERR_CUDA, L->err);
      levels[P] = std::move(L);
    }
    return true;
  }

  bool set_state_host(const double *Uh) {
    size_t count = (size_t)nS * E * nF;
    if (cudaMemcpyAsync(U, Uh, count * sizeof(double), cudaMemcpyHostToDevice, stream) != cudaSuccess)
      return fail(FR_ERR_CUDA, "cudaMemcpy H2D failed");
    if (mixed) split_state();
    extrapolate();
    if (in.dtType != 0) {  // solver::initializeSolution, solver.cpp:1932-1938
      wavesp_init();
      launches++;
    }
    stateSet = true;
    return cuda_ok("set_state");
  }

  // restrict_pmg (multigrid.cpp:315-345): U and divF[0] to the next coarser level
  void restrict_to(fr_case &C) {
    const long long N = (long long)C.E * C.nF;
    frk::launch_apply_op(restrictOp, U, C.U, N, 1.0, 0.0, stream);
    frk::launch_apply_op(restrictOp, divF[0], C.divF[0], N, 1.0, 0.0, stream);
    C.fptsFresh = false;
    launches += 2;
  }
  // precision form: the state restricted in FP64 from the joined state and
  // split again on the coarse level; the FP32 residual restricted in FP32
  void restrict_to32(fr_case &C) {
    const long long N = (long long)C.E * C.nF;
    join_state();
    frk::launch_apply_op(restrictOp, U, C.U, N, 1.0, 0.0, stream);
    C.split_state();
    frk::launch_apply_op_t<float>(restrictOp, f32.divF[0], C.f32.divF[0], N, stream);
    C.fptsFresh = false;
    launches += 4;
  }
  // prolong_err (multigrid.cpp:347-364): finer U += prolong(corr)
  void prolong_to(fr_case &F) {
    frk::launch_apply_op(prolongOp, corrPmg, F.U, (long long)E * nF, 1.0, 1.0, stream);
    F.fptsFresh = false;
    launches++;
  }

  // multiGrid::cycle (multigrid.cpp:169-313) for this (finest) level
  // multiGrid::cycle in the precision form: the smoothing stages run in FP32
  // with the source term in FP32; the restriction of the state, the source
  // term, the saved coarse solution, the correction and its prolongation run
  // in FP64 on the joined state (join/split around each transfer)
  bool pmg_cycle32() {
    if (!calc_residual(0)) return false;
    restrict_to32(*levels[in.order - 1]);
    for (int P = in.order - 1; P >= in.lowOrder; P--) {
      fr_case &L = *levels[P];
      const long long n = (long long)L.nS * L.E * L.nF;
      // compute_source_term (multigrid.cpp:366-384): restricted residual
      // minus the coarse level's own
      frk::launch_widen(n, L.f32.divF[0], L.src, stream);
      if (!L.calc_residual(0)) return fail(FR_ERR_CUDA, L.err);
      frk::launch_widen(n, L.f32.divF[0], L.corrPmg, stream);
      frk::launch_add(n, L.src, L.src, L.corrPmg, -1.0, stream);
      frk::launch_narrow(n, L.src, L.src32, stream);
      L.join_state();
      cudaMemcpyAsync(L.sol, L.U, n * sizeof(double), cudaMemcpyDeviceToDevice, stream);
      L.launches += 5;
      for (int st = 0; st < in.smoothSteps; st++)
        if (!L.update(true)) return fail(FR_ERR_CUDA, L.err);
      if (P - 1 >= in.lowOrder) {
        if (!L.calc_residual(0)) return fail(FR_ERR_CUDA, L.err);
        frk::launch_add32(n, L.f32.divF[0], L.f32.divF[0], L.src32, 1.0, stream);
        L.launches++;
        L.restrict_to32(*levels[P - 1]);
      }
    }
    for (int P = in.lowOrder; P <= in.order - 1; P++) {
      fr_case &L = *levels[P];
      const long long n = (long long)L.nS * L.E * L.nF;
      for (int st = 0; st < in.smoothSteps; st++)
        if (!L.update(true)) return fail(FR_ERR_CUDA, L.err);
      L.join_state();
      frk::launch_add(n, L.corrPmg, L.U, L.sol, -1.0, stream);
      fr_case &F = P < in.order - 1 ? *levels[P + 1] : *this;
      F.join_state();
      L.prolong_to(F);
      F.split_state();
      L.launches += 4;
    }
    return cuda_ok("pmg_cycle");
  }

  bool pmg_cycle() {
    if (!in.PMG || levels.empty()) return fail(FR_ERR_STATE, "no P-multigrid levels (PMG 0)");
    if (mixed) return pmg_cycle32();
    const long long nU = (long long)nS * E * nF;
    if (!calc_residual(0)) return false;
    restrict_to(*levels[in.order - 1]);
    for (int P = in.order - 1; P >= in.lowOrder; P--) {
      fr_case &L = *levels[P];
      const long long n = (long long)L.nS * L.E * L.nF;
      // compute_source_term (multigrid.cpp:366-384)
      cudaMemcpyAsync(L.src, L.divF[0], n * sizeof(double), cudaMemcpyDeviceToDevice, stream);
      if (!L.calc_residual(0)) return fail(FR_ERR_CUDA, L.err);
      frk::launch_add(n, L.src, L.src, L.divF[0], -1.0, stream);
      cudaMemcpyAsync(L.sol, L.U, n * sizeof(double), cudaMemcpyDeviceToDevice, stream);
      L.launches++;
      for (int st = 0; st < in.smoothSteps; st++)
        if (!L.update(true)) return fail(FR_ERR_CUDA, L.err);
      if (P - 1 >= in.lowOrder) {
        if (!L.calc_residual(0)) return fail(FR_ERR_CUDA, L.err);
        frk::launch_add(n, L.divF[0], L.divF[0], L.src, 1.0, stream);
        L.launches++;
        L.restrict_to(*levels[P - 1]);
      }
    }
    for (int P = in.lowOrder; P <= in.order - 1; P++) {
      fr_case &L = *levels[P];
      const long long n = (long long)L.nS * L.E * L.nF;
      for (int st = 0; st < in.smoothSteps; st++)
        if (!L.update(true)) return fail(FR_ERR_CUDA, L.err);
      frk::launch_add(n, L.corrPmg, L.U, L.sol, -1.0, stream);
      L.launches++;
      if (P < in.order - 1)
        L.prolong_to(*levels[P + 1]);
      else
        L.prolong_to(*this);
    }
    (void)nU;
    return cuda_ok("pmg_cycle");
  }

  long long total_launches() const {
    long long n = launches;
    for (auto &L : levels)
      if (L) n += L->total_launches();
    return n;
  }

  // Mesh, faces, metrics and operators on the host (no device needed).
  bool setup_host() {
    if (opts.mu_override) in.mu_inf = opts.mu_inf;
    nDims = in.nDims;
    nF = in.nFields;
    nRK = in.nRKSteps;
    std::string e;
    if (!fr::build_faces(mesh, in.order, in.sptsTypeQuad, faces, e)) return fail(FR_ERR_SETUP, e);
    if (!fr::build_geometry(mesh, in.order, in.sptsTypeQuad, geo, e)) return fail(FR_ERR_SETUP, e);
    fr::build_operators(nDims, in.order, in.sptsTypeQuad, in.vcjhSchemeQuad, op);
    nS = op.nSpts;
    nFp = op.nFpts;
    E = mesh.nEles;
    nPF = nDims == 2 ? in.order + 1 : (in.order + 1) * (in.order + 1);
    return true;
  }

  bool setup_motion() {
    if (mixed) return fail(FR_ERR_UNSUPPORTED, "moving meshes run in the plain form, not the precision form");
    auto &a = mo.a;
    const int nd = nDims;
    a.type = in.motion;
    a.nDims = nd;
    a.nVerts = mesh.nVerts;
    a.E = E;
    a.nS = nS;
    a.nFp = nFp;
    a.nNodes = mesh.nNodes;
    a.time = timeAcc;
    a.dt = dt;
    // motion 1 scales by the periodic lengths (src/geo.cpp:2737-2738)
    a.DX = mesh.period[0];
    a.DY = mesh.period[1];
    a.Ax = in.moveAx;
    a.Ay = in.moveAy;
    a.Fx = in.moveFx;
    a.Fy = in.moveFy;
    a.Ar = in.moveAr;
    a.Fr = in.moveFr;
    std::vector<double> xv0(mesh.xv.begin(), mesh.xv.begin() + (size_t)mesh.nVerts * nd);
    double *dxv0, *dxv, *dgv;
    if (!upload(dxv0, xv0) || !alloc(dxv, xv0.size()) || !alloc(dgv, xv0.size())) return false;
    a.xv0 = dxv0;
    a.xv = dxv;
    a.gv = dgv;
    if (in.motion == 5) {  // spherical coordinates of the initial vertices (src/geo.cpp:208-216)
      std::vector<double> rv((size_t)mesh.nVerts * 3);
      for (int i = 0; i < mesh.nVerts; i++) {
        const double x = xv0[(size_t)i * 3], y = xv0[(size_t)i * 3 + 1], z = xv0[(size_t)i * 3 + 2];
        rv[(size_t)i * 3] = std::sqrt(x * x + y * y + z * z);
        rv[(size_t)i * 3 + 1] = std::atan2(y, x);
        rv[(size_t)i * 3 + 2] = std::acos(z / rv[(size_t)i * 3]);
      }
      double *drv;
      if (!upload(drv, rv)) return false;
      a.rv0 = drv;
    }
    int *dc2v;
    if (!upload(dc2v, mesh.c2v)) return false;
    a.c2v = dc2v;
    auto loc = fr::loc_spts(nd, in.order, in.sptsTypeQuad);
    auto lf = fr::loc_fpts(nd, in.order, in.sptsTypeQuad);
    loc.insert(loc.end(), lf.begin(), lf.end());
    std::vector<double> N, dN;
    std::string e;
    if (!fr::shape_tables(nd, mesh.nNodes, loc, N, dN, e)) return fail(FR_ERR_SETUP, e);
    double *dNs, *ddN, *dtn, *dJ, *dgs, *dgf;
    if (!upload(dNs, N) || !upload(ddN, dN) || !upload(dtn, op.tNorm) || !alloc(dJ, (size_t)nd * nS * E * nd) ||
        !alloc(dgs, (size_t)nS * E * nd) || !alloc(dgf, (size_t)nFp * E * nd))
      return false;
    a.shape = dNs;
    a.dshape = ddN;
    a.tNorm = dtn;
    a.Jac = dJ;
    a.gVs = dgs;
    a.gVf = dgf;
    a.JGinv = JGinv;
    a.detJ = detJ;
    a.norm = norm;
    a.dA = dA;
    std::vector<double> G;
    for (int d = 0; d < nd; d++) G.insert(G.end(), op.grad[d].begin(), op.grad[d].end());
    double *dG, *dX, *dC;
    if (!upload(dG, G) || !upload(dX, op.ext) || !upload(dC, op.corr)) return false;
    a.opGrad = dG;
    a.opExt = dX;
    a.opCorr = dC;
    if (!alloc(mo.err, 1) || !alloc(mo.F, (size_t)nd * nS * E * nF) || !alloc(mo.disFn, (size_t)nFp * E * nF))
      return false;
    a.err = mo.err;
    mo.on = true;
    // solver::initializeSolution places the mesh at the current time before
    // the initial condition (src/solver.cpp:1902-1904); the metrics are those
    // of the mesh as set up, which a rigid translation (motion 4) keeps
    frk::launch_move_vertices(mo.a, 0.0, stream);
    frk::launch_motion_geometry(mo.a, true, stream);
    frk::launch_face_refresh(ft, nDims, norm, dA, stream);
    return cuda_ok("motion setup");
  }

  // solver::moveMesh (src/solver.cpp:1168-1246, non-overset branch): the
  // vertices at time + dt * rkVal, then grid velocities and (except for a
  // rigid translation, motion 4) the metrics and the face table's copies.
  void move_mesh(double rkVal) {
    frk::launch_move_vertices(mo.a, rkVal, stream);
    frk::launch_motion_geometry(mo.a, in.motion != 4, stream);
    launches += 2;
    if (in.motion != 4) {
      frk::launch_face_refresh(ft, nDims, norm, dA, stream);
      launches++;
    }
  }

  // calcResidual on the moving mesh (src/solver.cpp:366-445 with motion):
  // extrapolation, common flux with grid velocity, chain-rule divergence,
  // correction; divF into divF[step].
  void residual_motion(int step) {
    extrapolate();
    frk::launch_faces_motion(nDims, ft, Ufpts, Fn, waveSp, mo.a.gVf, ph, stream);
    frk::launch_motion_residual(mo.a, U, Fn, in.gamma, mo.F, mo.disFn, divF[step], stream);
    launches += 5;
    fptsFresh = false;
  }

  // solver::update with motion (src/solver.cpp:319-363): the metrics move
  // with every stage, and a standard RK step combines its stored stage
  // residuals at the end with the last stage's metrics.  A P-multigrid level
  // moves its own mesh with its own time, which its updates advance
  // (multigrid.cpp:130-135: every level solves with its own copy of the
  // inputs), and adds its source term to each stage residual.
  bool update_motion(bool pmgSource) {
    const double *eDt = in.dtType == 2 ? eleDt : nullptr;
    const double *srcU = pmgSource ? src : nullptr;
    const long long nSE = (long long)nS * E;
    const bool jameson = in.timeType >= 5;
    for (int step = 0; step < nRK - 1; step++) {
      if (step == 0 && in.dtType != 0) calc_dt_dev();
      move_mesh(in.RKa[step]);
      if (step == 0) cudaMemcpyAsync(U0, U, (size_t)nSE * nF * sizeof(double), cudaMemcpyDeviceToDevice, stream);
      residual_motion(step);
      frk::launch_motion_step_a(nSE, nF, E, U0, divF[step], srcU, detJ, dt, eDt, in.RKa[step + 1], U, stream);
      launches++;
    }
    move_mesh(in.RKa[nRK - 1]);
    residual_motion(nRK - 1);
    if (!jameson) {
      if (nRK == 1 && in.dtType != 0) calc_dt_dev();
      frk::MotionStages stg;
      stg.n = nRK;
      for (int s2 = 0; s2 < nRK; s2++) {
        stg.divF[s2] = divF[s2];
        stg.rkb[s2] = in.RKb[s2];
      }
      frk::launch_motion_step_b(nSE, nF, E, nRK > 1 ? U0 : U, stg, srcU, detJ, dt, eDt, U, stream);
    } else {
      frk::launch_motion_step_a(nSE, nF, E, U0, divF[nRK - 1], srcU, detJ, dt, eDt, in.RKa[nRK], U, stream);
    }
    frk::launch_add_time(dt, timeAcc, stream);
    launches += 2;
    fptsFresh = false;
    return cuda_ok("update (moving mesh)");
  }

  // Tensor-product tables of the dense operators, used only if every dense
  // entry is reproduced bitwise (reference operators: operators.cpp:112-141,
  // 596-655, 715-824).
  bool build_tp() {
    if (!frk::tp_supported(nDims, in.order)) return false;
    const int n = in.order + 1;
    auto p1 = fr::pts1d(in.sptsTypeQuad, in.order);
    auto fp = fr::loc_fpts(nDims, in.order, in.sptsTypeQuad);
    auto ijk = [&](int sp, int *id) {
      id[0] = sp % n;
      id[1] = nDims > 1 ? (sp / n) % n : 0;
      id[2] = nDims > 2 ? sp / (n * n) : 0;
    };
    auto strideOf = [&](int d) { return d == 0 ? 1 : (d == 1 ? n : n * n); };
    std::vector<double> D((size_t)n * n);
    for (int i = 0; i < n; i++)
      for (int m = 0; m < n; m++) D[(size_t)i * n + m] = op.grad[0][(size_t)i * nS + m];
    for (int d = 0; d < nDims; d++)
      for (int sp = 0; sp < nS; sp++) {
        int a[3];
        ijk(sp, a);
        int base = sp - a[d] * strideOf(d);
        for (int c = 0; c < nS; c++) {
          int b[3];
          ijk(c, b);
          bool on = true;
          for (int q = 0; q < nDims; q++)
            if (q != d && b[q] != a[q]) on = false;
          double ex = on ? D[(size_t)a[d] * n + b[d]] : 0.0;
          if (on && c != base + b[d] * strideOf(d)) return false;
          if (op.grad[d][(size_t)sp * nS + c] != ex) return false;
        }
      }
    std::vector<int> fBase(nFp), fDn(nFp), fSide(nFp);
    std::vector<double> E1(2 * n, 0.0), EF(2 * n, 0.0);
    bool have[2] = {false, false};
    for (int f = 0; f < nFp; f++) {
      int dn = -1;
      for (int d = 0; d < nDims; d++)
        if (op.tNorm[(size_t)f * nDims + d] != 0.0) dn = d;
      if (dn < 0) return false;
      int side = op.tNorm[(size_t)f * nDims + dn] > 0 ? 1 : 0;
      int id[3] = {0, 0, 0};
      for (int d = 0; d < nDims; d++) {
        if (d == dn) continue;
        int hit = -1;
        for (int i = 0; i < n; i++)
          if (fp[f][d] == p1[i]) hit = i;
        if (hit < 0) return false;
        id[d] = hit;
      }
      int base = id[0] + n * id[1] + n * n * id[2];
      fBase[f] = base;
      fDn[f] = dn;
      fSide[f] = side;
      if (!have[side]) {
        for (int m = 0; m < n; m++) {
          E1[side * n + m] = op.ext[(size_t)f * nS + base + m * strideOf(dn)];
          EF[side * n + m] = op.extFn[dn][(size_t)f * nS + base + m * strideOf(dn)];
        }
        have[side] = true;
      }
      for (int c = 0; c < nS; c++) {
        int b[3];
        ijk(c, b);
        bool on = true;
        for (int d = 0; d < nDims; d++)
          if (d != dn && b[d] != id[d]) on = false;
        if (op.ext[(size_t)f * nS + c] != (on ? E1[side * n + b[dn]] : 0.0)) return false;
        for (int d = 0; d < nDims; d++)
          if (op.extFn[d][(size_t)f * nS + c] != (on && d == dn ? EF[side * n + b[dn]] : 0.0)) return false;
      }
    }
    // the two flux points at the ends of each line (side 0 first), so that
    // one pass over a line's points extrapolates to both
    std::vector<int> pair;
    for (int f = 0; f < nFp; f++) {
      if (fSide[f] != 0) continue;
      int g = -1;
      for (int h = 0; h < nFp; h++)
        if (fSide[h] == 1 && fBase[h] == fBase[f] && fDn[h] == fDn[f]) g = h;
      if (g < 0) return false;
      pair.push_back(f | g << 16);
    }
    if ((int)pair.size() * 2 != nFp) return false;
    const int nFaces = 2 * nDims;
    std::vector<int> cF((size_t)nS * nFaces);
    std::vector<double> cV((size_t)nS * nFaces);
    for (int sp = 0; sp < nS; sp++) {
      int a[3];
      ijk(sp, a);
      for (int fc = 0; fc < nFaces; fc++) {
        int hit = -1;
        for (int j = 0; j < nPF; j++) {
          int f = fc * nPF + j;
          if (fBase[f] == sp - a[fDn[f]] * strideOf(fDn[f])) hit = f;
        }
        if (hit < 0) return false;
        cF[(size_t)sp * nFaces + fc] = hit;
        cV[(size_t)sp * nFaces + fc] = op.corr[(size_t)sp * nFp + hit];
      }
      for (int c = 0; c < nFp; c++) {
        bool used = false;
        for (int fc = 0; fc < nFaces; fc++)
          if (cF[(size_t)sp * nFaces + fc] == c) used = true;
        if (!used && op.corr[(size_t)sp * nFp + c] != 0.0) return false;
      }
      // ascending flux-point order of the dense row
      for (int fc = 1; fc < nFaces; fc++)
        if (cF[(size_t)sp * nFaces + fc] <= cF[(size_t)sp * nFaces + fc - 1]) return false;
    }
    // the correction values as a function of the side of the face and the
    // point's index along its normal (tensor product), checked bit for bit:
    // the 3-D element kernels apply the correction line by line
    std::vector<double> LC(2 * n, 0.0);
    std::vector<char> seen(2 * n, 0);
    for (int sp = 0; sp < nS; sp++) {
      int a[3];
      ijk(sp, a);
      for (int fc = 0; fc < nFaces; fc++) {
        const int f = cF[(size_t)sp * nFaces + fc];
        const int k = fSide[f] * n + a[fDn[f]];
        const double v = cV[(size_t)sp * nFaces + fc];
        if (!seen[k]) {
          LC[k] = v;
          seen[k] = 1;
        } else if (LC[k] != v) {
          return false;
        }
      }
    }
    double *dD, *dE1, *dEF, *dcV, *dLC;
    int *dfB, *dfD, *dfS, *dcF, *dLP;
    if (!upload(dD, D) || !upload(dE1, E1) || !upload(dEF, EF) || !upload(dfB, fBase) || !upload(dfD, fDn) ||
        !upload(dfS, fSide) || !upload(dcF, cF) || !upload(dcV, cV) || !upload(dLP, pair) || !upload(dLC, LC))
      return false;
    tp.linePair = f32.tp.linePair = dLP;
    tp.lineCorr = dLC;
    tp.D = dD;
    tp.E1 = dE1;
    tp.EFn1 = dEF;
    tp.fptBase = f32.tp.fptBase = dfB;
    tp.fptDn = f32.tp.fptDn = dfD;
    tp.fptSide = f32.tp.fptSide = dfS;
    tp.corrFpt = f32.tp.corrFpt = dcF;
    tp.corrVal = dcV;
    if (mixed) {
      float *fD, *fE1, *fEF, *fcV, *fLC;
      if (!upload(fD, narrow(D)) || !upload(fE1, narrow(E1)) || !upload(fEF, narrow(EF)) || !upload(fcV, narrow(cV)) ||
          !upload(fLC, narrow(LC)))
        return false;
      f32.tp.D = fD;
      f32.tp.E1 = fE1;
      f32.tp.EFn1 = fEF;
      f32.tp.corrVal = fcV;
      f32.tp.lineCorr = fLC;
    }
    return true;
  }

  static std::vector<float> narrow(const std::vector<double> &v) {
    std::vector<float> o(v.size());
    for (size_t i = 0; i < v.size(); i++) o[i] = (float)v[i];
    return o;
  }

  static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    if (!encode) {
      void *fn = nullptr;
      cudaDriverEntryPointQueryResult q;
      if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
          q != cudaDriverEntryPointSuccess || !fn)
        return nullptr;
      encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
    }
    return encode;
  }

  // Tile-shape autotuner of the precision form: times the TMA element stage
  // (an intermediate RK stage, the common case) for every tile variant on
  // this case's own arrays and keeps the fastest.  Runs at setup, before any
  // state exists; the arrays it touched are cleared afterwards.  Every
  // variant computes each point with the same operations, so the choice
  // changes the speed only, never the result.
  bool autotune_tiles() {
    const bool tc = frk::tc_supported(nDims, in.order) && !opts.no_tensor_cores;
    if (tc && !f32.tcOps) {
      const double *g[3] = {op.grad[0].data(), op.grad[1].data(), nDims == 3 ? op.grad[2].data() : nullptr};
      const double *x[3] = {op.extFn[0].data(), op.extFn[1].data(), nDims == 3 ? op.extFn[2].data() : nullptr};
      std::vector<float> blob;
      if (!frk::tc_pack_ops(nDims, in.order, g, x, op.corr.data(), op.ext.data(), blob) || !upload(f32.tcOps, blob))
        return fail(FR_ERR_CUDA, "tensor-core operator upload");
    }
    const int nv = frk::tma_variants(true) + (tc ? 1 : 0);
    int forced = opts.tile_variant;
    f32.tuneMs.assign(nv, -1.0f);
    if (forced >= nv) return fail(FR_ERR_ARG, "tile_variant out of range");
    // small cases: launches of a few microseconds time as noise, so the
    // choice is fixed (the first shape) and identical cases stay identical
    if (forced < 0 && (long long)nS * E < kTuneMinPoints) forced = 0;
    int best = -1;
    float bestMs = 0.0f;
    const int tpEB = EB;
    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)
      return fail(FR_ERR_CUDA, "event create");
    for (int v = 0; v < nv; v++) {
      if (forced >= 0 && v != forced) continue;
      bool dup = false;  // CUDA-core variants that clamp to the same tile are timed once
      for (int w = 0; w < v && v < frk::tma_variants(true); w++)
        if (frk::tma_elems_per_block<float>(nDims, in.order, w) == frk::tma_elems_per_block<float>(nDims, in.order, v))
          dup = true;
      if (dup && forced < 0) continue;
      if (!build_tma32(v)) continue;
      f32.variant = v;
      EB = frk::tma_elems_per_block<float>(nDims, in.order, v);
      frk::ElemArgsT<float> a = elem_args32();
      a.mode = frk::MODE_RK_STAGE;
      a.stage = 1;
      a.Ufpts_out = f32.Ufpts;
      for (int i = 0; i < 2; i++) launch_tma32(a, v);
      cudaEventRecord(e0, stream);
      const int reps = 5;
      for (int i = 0; i < reps; i++) launch_tma32(a, v);
      cudaEventRecord(e1, stream);
      if (cudaEventSynchronize(e1) != cudaSuccess) break;
      float ms = 0.0f;
      cudaEventElapsedTime(&ms, e0, e1);
      ms /= reps;
      f32.tuneMs[v] = ms;
      // the tensor-core variant differs from the CUDA-core ones by FP32
      // round-off: it must win clearly, not by timing noise
      const bool tcv = v == frk::tma_variants(true);
      if (best < 0 || (tcv ? ms < 0.9f * bestMs : ms < bestMs)) {
        best = v;
        bestMs = ms;
      }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (!cuda_ok("tile autotune")) return false;
    if (!sync()) return false;
    if (best < 0) {  // no TMA variant applies: tensor-product kernel
      EB = tpEB;
      return true;
    }
    if (!build_tma32(best)) return fail(FR_ERR_CUDA, "tensor map");
    f32.variant = best;
    f32.useTma = true;
    EB = frk::tma_elems_per_block<float>(nDims, in.order, best);
    const size_t nU = (size_t)nS * E * nF, nUf = (size_t)nFp * E * nF;
    for (float *p : {f32.U, f32.U0, f32.acc, f32.comp}) cudaMemsetAsync(p, 0, nU * sizeof(float), stream);
    cudaMemsetAsync(f32.Ufpts, 0, nUf * sizeof(float), stream);
    cudaMemsetAsync(devErr, 0, sizeof(unsigned), stream);
    return sync();
  }

  // The metric arrays as the TMA element kernels read them: every row pitch
  // of a tensor map must be a multiple of 16 bytes, so when E is not a
  // multiple of `align` elements, copies of detJ and JGinv with the element
  // axis padded to Ep (zeros in the padding) serve the tensor maps.
  template <typename T>
  bool tma_metrics(int align, T *det, T *jg, T *&detOut, T *&jgOut, int &Ep) {
    Ep = (E + align - 1) / align * align;
    detOut = det;
    jgOut = jg;
    if (Ep == E) return true;
    std::vector<T> d((size_t)nS * Ep, T(0)), j((size_t)nDims * nS * Ep * nDims, T(0));
    for (int s = 0; s < nS; s++)
      for (int e = 0; e < E; e++) d[(size_t)s * Ep + e] = (T)geo.detJac_spts[(size_t)s * E + e];
    for (int a = 0; a < nDims * nS; a++)
      for (int e = 0; e < E; e++)
        for (int b = 0; b < nDims; b++)
          j[((size_t)a * Ep + e) * nDims + b] = (T)geo.JGinv_spts[((size_t)a * E + e) * nDims + b];
    return upload(detOut, d) && upload(jgOut, j);
  }

  // TMA descriptors for the tile copies of a TMA element kernel: element
  // block eb, element type T.  State rows need E*nF*sizeof(T) to be a
  // multiple of 16 bytes (2-D always; 3-D E even in FP64, E a multiple of 4
  // in FP32); the metrics use padded copies where needed.
  template <typename T>
  bool build_maps(frk::TmaMaps &t, int eb, T *u, T *u0, T *ac, T *cmp, T *fn, T *uf, T *det, T *jg,
                  T *&detPad, T *&jgPad, T *dus = nullptr, T *duc = nullptr, T *duf = nullptr) {
    const int align = 16 / (int)sizeof(T);
    if ((E * nF) % align != 0 || nS > 256 || nFp > 256 || eb <= 0 || (eb * nF) % align != 0 ||
        (eb * nDims) % align != 0 || eb % align != 0)
      return false;
    auto encode = tensor_map_encoder();
    if (!encode) return false;
    const CUtensorMapDataType ty = sizeof(T) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    auto map2 = [&](CUtensorMap *m, void *p, cuuint64_t inner, cuuint64_t outer, cuuint64_t pitch, cuuint32_t bi,
                    cuuint32_t bo) {
      cuuint64_t dims[2] = {inner, outer};
      cuuint64_t str[1] = {pitch * sizeof(T)};
      cuuint32_t box[2] = {bi, bo};
      cuuint32_t es[2] = {1, 1};
      return encode(m, ty, 2, p, dims, str, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
    };
    int Ep = E;
    if (!detPad && !tma_metrics<T>(align, det, jg, detPad, jgPad, Ep)) return false;
    Ep = (E + align - 1) / align * align;
    const cuuint64_t rowU = (cuuint64_t)E * nF;
    bool ok = map2(&t.U, u, rowU, nS, rowU, eb * nF, nS) && map2(&t.Fn, fn, rowU, nFp, rowU, eb * nF, nFp) &&
              map2(&t.Ufpts, uf, rowU, nFp, rowU, eb * nF, nFp) && map2(&t.det, detPad, E, nS, Ep, eb, nS);
    if (u0) ok = ok && map2(&t.U0, u0, rowU, nS, rowU, eb * nF, nS);
    if (ac) ok = ok && map2(&t.acc, ac, rowU, nS, rowU, eb * nF, nS);
    if (cmp) ok = ok && map2(&t.comp, cmp, rowU, nS, rowU, eb * nF, nS);
    if (!ok) return false;
    auto map3 = [&](CUtensorMap *m, void *p, cuuint64_t d0, cuuint64_t d1, cuuint64_t d2, cuuint64_t pitch0,
                    cuuint32_t b0, cuuint32_t b1, cuuint32_t b2) {
      cuuint64_t dims[3] = {d0, d1, d2};
      cuuint64_t str[2] = {pitch0 * sizeof(T), pitch0 * d1 * sizeof(T)};
      cuuint32_t box[3] = {b0, b1, b2};
      cuuint32_t es[3] = {1, 1, 1};
      return encode(m, ty, 3, p, dims, str, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
    };
    if (!map3(&t.J, jgPad, (cuuint64_t)E * nDims, nS, nDims, (cuuint64_t)Ep * nDims, eb * nDims, nS, nDims))
      return false;
    // viscous: gradients [nDims][points][E*nF], jumps [nFp][E*nF]
    if (dus && !map3(&t.dUs, dus, rowU, nS, nDims, rowU, eb * nF, nS, nDims)) return false;
    if (duf && !map3(&t.dUf, duf, rowU, nFp, nDims, rowU, eb * nF, nFp, nDims)) return false;
    if (duc && !map2(&t.dUc, duc, rowU, nFp, rowU, eb * nF, nFp)) return false;
    return true;
  }
  double *detTma = nullptr, *jgTma = nullptr;
  float *detTma32 = nullptr, *jgTma32 = nullptr;

  bool build_tma(int v) {
    return build_maps<double>(tm, frk::tma_elems_per_block<double>(nDims, in.order, v), U, U0, acc, nullptr, Fn,
                              Ufpts, detJ, JGinv, detTma, jgTma, dUs, dUc, dUf);
  }

  // The plain form's tile autotuner: the same timing as autotune_tiles on
  // the FP64 arrays; all variants give bit-identical results.
  bool autotune_tiles64() {
    const int nv = frk::tma_variants(false);
    int forced = opts.tile_variant;
    if (forced >= nv) return fail(FR_ERR_ARG, "tile_variant out of range for the plain form");
    if (forced < 0 && (long long)nS * E < kTuneMinPoints) forced = 0;  // small: fixed choice
    tuneMs64.assign(nv, -1.0f);
    int best = -1;
    float bestMs = 0.0f;
    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)
      return fail(FR_ERR_CUDA, "event create");
    for (int v = 0; v < nv; v++) {
      if (forced >= 0 && v != forced) continue;
      bool dup = false;
      for (int w = 0; w < v; w++)
        if (frk::tma_elems_per_block<double>(nDims, in.order, w) == frk::tma_elems_per_block<double>(nDims, in.order, v))
          dup = true;
      if (dup && forced < 0) continue;
      if (!build_tma(v)) continue;
      frk::ElemArgs a = elem_args();
      a.mode = frk::MODE_RK_STAGE;
      a.stage = 1;
      a.Ufpts_out = Ufpts;
      for (int i = 0; i < 2; i++) frk::launch_element_stage_tma<double>(nDims, in.order, a, tp, tm, stream, v);
      cudaEventRecord(e0, stream);
      const int reps = 5;
      for (int i = 0; i < reps; i++) frk::launch_element_stage_tma<double>(nDims, in.order, a, tp, tm, stream, v);
      cudaEventRecord(e1, stream);
      if (cudaEventSynchronize(e1) != cudaSuccess) break;
      float ms = 0.0f;
      cudaEventElapsedTime(&ms, e0, e1);
      tuneMs64[v] = ms / reps;
      if (best < 0 || tuneMs64[v] < bestMs) {
        best = v;
        bestMs = tuneMs64[v];
      }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (!cuda_ok("tile autotune") || !sync()) return false;
    if (best < 0) best = 0;
    if (!build_tma(best)) return fail(FR_ERR_CUDA, "tensor map");
    variant64 = best;
    const size_t nU = (size_t)nS * E * nF, nUf = (size_t)nFp * E * nF;
    for (double *p : {U, U0, acc}) cudaMemsetAsync(p, 0, nU * sizeof(double), stream);
    cudaMemsetAsync(Ufpts, 0, nUf * sizeof(double), stream);
    cudaMemsetAsync(devErr, 0, sizeof(unsigned), stream);
    return sync();
  }
  bool build_tma32(int v) {
    return build_maps<float>(f32.tm, frk::tma_elems_per_block<float>(nDims, in.order, v), f32.U, f32.U0, f32.acc,
                             f32.comp, f32.Fn, f32.Ufpts, f32.detJ, f32.JGinv, detTma32, jgTma32, f32.dUs, f32.dUc,
                             f32.dUf);
  }

  // Merge the host data of several same-order cases along the element axis
  // (face element indices shifted, metric arrays concatenated), then set up
  // the device side and copy the members' states and time steps in.
  bool merge_from(const std::vector<fr_case *> &ms, const fr_setup_opts &o) {
    opts = o;
    opts.debug_arrays = 0;
    mixed = o.precision == FR_PREC_MIXED;
    const fr_case &f = *ms[0];
    in = f.in;
    nDims = f.nDims;
    nF = f.nF;
    nRK = f.nRK;
    nS = f.nS;
    nFp = f.nFp;
    nPF = f.nPF;
    op = f.op;
    perElementDt = true;
    E = 0;
    std::vector<int> off;
    for (auto *m : ms) {
      off.push_back(E);
      E += m->E;
    }
    mesh.nDims = nDims;
    mesh.nEles = E;
    auto cat = [&](std::vector<double> fr::Geometry::*field, size_t A, size_t B) {
      std::vector<double> out(A * (size_t)E * B);
      for (size_t a = 0; a < A; a++)
        for (size_t k = 0; k < ms.size(); k++) {
          const auto &src = ms[k]->geo.*field;
          const size_t Em = ms[k]->E;
          std::copy(src.begin() + a * Em * B, src.begin() + (a + 1) * Em * B,
                    out.begin() + (a * (size_t)E + off[k]) * B);
        }
      geo.*field = std::move(out);
    };
    cat(&fr::Geometry::pos_spts, nS, nDims);
    cat(&fr::Geometry::pos_fpts, nFp, nDims);
    cat(&fr::Geometry::detJac_spts, nS, 1);
    cat(&fr::Geometry::detJac_fpts, nFp, 1);
    cat(&fr::Geometry::JGinv_spts, (size_t)nDims * nS, nDims);
    cat(&fr::Geometry::norm_fpts, nFp, nDims);
    cat(&fr::Geometry::dA_fpts, nFp, 1);
    faces.clear();
    for (size_t k = 0; k < ms.size(); k++)
      for (auto fc : ms[k]->faces) {
        fc.eL += off[k];
        if (fc.eR >= 0) fc.eR += off[k];
        faces.push_back(std::move(fc));
      }
    if (cudaSetDevice(o.device) != cudaSuccess) return fail(FR_ERR_CUDA, "cudaSetDevice failed");
    if (cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) != cudaSuccess)
      return fail(FR_ERR_CUDA, "stream create");
    ownStream = true;
    ownedStream = stream;
    if (!setup_device()) return false;
    std::vector<double> edt(E);
    for (size_t k = 0; k < ms.size(); k++) {
      fr_case &m = *ms[k];
      if (!m.sync()) return fail(FR_ERR_CUDA, m.err);
      for (int e = 0; e < m.E; e++) edt[off[k] + e] = m.hostDt;
      if (!mixed) {
        if (!copy_rows(U, E, off[k], m.U, m.E, 0)) return fail(FR_ERR_CUDA, "state gather failed");
      } else if (!copy_rows(f32.U, E, off[k], m.f32.U, m.E, 0) || !copy_rows(f32.comp, E, off[k], m.f32.comp, m.E, 0)) {
        return fail(FR_ERR_CUDA, "state gather failed");
      }
    }
    if (cudaMemcpyAsync(eleDt, edt.data(), E * sizeof(double), cudaMemcpyHostToDevice, stream) != cudaSuccess)
      return fail(FR_ERR_CUDA, "dt upload failed");
    extrapolate();
    stateSet = true;
    return sync();
  }

  // Copy a member's slice of this merged state back into the member case.
  bool scatter_to(fr_case &m, int offset) {
    if (!mixed) {
      if (!copy_rows(m.U, m.E, 0, U, E, offset)) return fail(FR_ERR_CUDA, "state scatter failed");
      if (!copy_rows(m.divF[0], m.E, 0, divF[0], E, offset)) return fail(FR_ERR_CUDA, "residual scatter failed");
    } else {
      if (!copy_rows(m.f32.U, m.E, 0, f32.U, E, offset) || !copy_rows(m.f32.comp, m.E, 0, f32.comp, E, offset))
        return fail(FR_ERR_CUDA, "state scatter failed");
      if (!copy_rows(m.f32.divF[0], m.E, 0, f32.divF[0], E, offset))
        return fail(FR_ERR_CUDA, "residual scatter failed");
    }
    m.fptsFresh = false;
    return true;
  }

  // Part r of a case split by the element partition `part` (fr_shard_*):
  // the part's elements (ascending global ids; local id = rank among them),
  // its metric arrays sliced from the whole case's, the faces between two of
  // its elements and its boundary faces, renumbered, and its cut face points
  // (a face whose other element is in another part): each with this part's
  // element as the left side, listed by peer part and, per peer, by face
  // (the whole case's face order) and by the face's left point order, the
  // order fr_shard_plan gives and both sides of a cut share.  Plain form,
  // inviscid, static mesh, no P-multigrid (the creator checks).
  bool split_from(const fr_case &full, const std::vector<int> &part, int r, cudaStream_t st) {
    opts = full.opts;
    opts.no_pdl = 1;  // parts run in one stream with copies between their kernels
    in = full.in;
    nDims = full.nDims;
    nF = full.nF;
    nRK = full.nRK;
    nS = full.nS;
    nFp = full.nFp;
    nPF = full.nPF;
    op = full.op;
    const int Ef = full.E;
    std::vector<int> owned, local(Ef, -1);
    for (int e = 0; e < Ef; e++)
      if (part[e] == r) {
        local[e] = (int)owned.size();
        owned.push_back(e);
      }
    E = (int)owned.size();
    if (E == 0) return fail(FR_ERR_ARG, "empty part");
    mesh.nDims = nDims;
    mesh.nEles = E;
    auto sel = [&](const std::vector<double> &src, size_t A, size_t B) {
      std::vector<double> out(A * (size_t)E * B);
      for (size_t a = 0; a < A; a++)
        for (int el = 0; el < E; el++)
          for (size_t b = 0; b < B; b++) out[(a * E + el) * B + b] = src[(a * Ef + owned[el]) * B + b];
      return out;
    };
    geo.pos_spts = sel(full.geo.pos_spts, nS, nDims);
    geo.pos_fpts = sel(full.geo.pos_fpts, nFp, nDims);
    geo.detJac_spts = sel(full.geo.detJac_spts, nS, 1);
    geo.detJac_fpts = sel(full.geo.detJac_fpts, nFp, 1);
    geo.JGinv_spts = sel(full.geo.JGinv_spts, (size_t)nDims * nS, nDims);
    geo.norm_fpts = sel(full.geo.norm_fpts, nFp, nDims);
    geo.dA_fpts = sel(full.geo.dA_fpts, nFp, 1);
    struct CutPt {
      int peer, slot, left;
    };
    std::vector<CutPt> cuts;
    faces.clear();
    for (const fr::Face &f : full.faces) {
      const bool mineL = part[f.eL] == r, mineR = f.eR >= 0 && part[f.eR] == r;
      if (f.eR < 0 || (mineL && mineR)) {
        if (!mineL) continue;
        fr::Face g = f;
        g.eL = local[f.eL];
        if (f.eR >= 0) g.eR = local[f.eR];
        faces.push_back(std::move(g));
      } else if (mineL || mineR) {
        for (int j = 0; j < nPF; j++) {
          if (mineL)
            cuts.push_back({part[f.eR], (f.locL * nPF + j) * E + local[f.eL], 1});
          else
            cuts.push_back({part[f.eL], f.fptR[j] * E + local[f.eR], 0});
        }
      }
    }
    std::stable_sort(cuts.begin(), cuts.end(), [](const CutPt &a, const CutPt &b) { return a.peer < b.peer; });
    stream = st;
    ownStream = false;
    if (!setup_device()) return false;
    if (!cuts.empty()) {
      const size_t n = cuts.size();
      std::vector<int> sl(n), lf(n);
      std::vector<double> nv(n * nDims), da(n);
      cutPeer.resize(n);
      for (size_t i = 0; i < n; i++) {
        sl[i] = cuts[i].slot;
        lf[i] = cuts[i].left;
        cutPeer[i] = cuts[i].peer;
        for (int d = 0; d < nDims; d++) nv[i * nDims + d] = geo.norm_fpts[(size_t)sl[i] * nDims + d];
        da[i] = geo.dA_fpts[sl[i]];
      }
      int *dsl, *dlf;
      double *dnv, *dda, *snd, *rcv;
      if (!upload(dsl, sl) || !upload(dlf, lf) || !upload(dnv, nv) || !upload(dda, da) || !alloc(snd, n * nF) ||
          !alloc(rcv, n * nF))
        return false;
      cut.n = (int)n;
      cut.slot = dsl;
      cut.left = dlf;
      cut.nrm = dnv;
      cut.dA = dda;
      cut.send = snd;
      cut.recv = rcv;
    }
    return sync();
  }

  // rows [nS] of m elements: dst[s][dOff..dOff+m) = src[s][sOff..sOff+m), all
  // fields, arrays of dE / sE elements per row
  template <typename T>
  bool copy_rows(T *dst, int dE, int dOff, const T *src, int sE, int sOff) {
    const int m = std::min(dE - dOff, sE - sOff);
    return cudaMemcpy2DAsync(dst + (size_t)dOff * nF, (size_t)dE * nF * sizeof(T), src + (size_t)sOff * nF,
                             (size_t)sE * nF * sizeof(T), (size_t)m * nF * sizeof(T), nS, cudaMemcpyDeviceToDevice,
                             stream) == cudaSuccess;
  }

  frk::ElemArgs elem_args() {
    frk::ElemArgs a;
    a.E = E;
    a.nS = nS;
    a.nFp = nFp;
    a.EB = EB;
    a.U = U;
    a.JGinv = JGinv;
    a.detJ = detJ;
    a.Fn = Fn;
    for (int d = 0; d < nDims; d++) {
      a.grad[d] = grad[d];
      a.extFn[d] = extFn[d];
    }
    a.corr = corr;
    a.ext = ext;
    a.nRK = nRK;
    a.dt = dt;
    a.eleDt = (in.dtType == 2 || perElementDt) ? eleDt : nullptr;
    a.U0 = U0;
    a.acc = acc;
    a.Uout = U;
    a.err = devErr;
    a.gamma = in.gamma;
    a.ph = ph;
    if (in.viscous) {
      a.dUs = dUs;
      a.dUsStride = (long long)nS * E * nF;
    }
    return a;
  }

  frk::ElemArgsT<float> elem_args32() {
    frk::ElemArgsT<float> a;
    a.E = E;
    a.nS = nS;
    a.nFp = nFp;
    a.EB = EB;
    a.U = f32.U;
    a.JGinv = f32.JGinv;
    a.detJ = f32.detJ;
    a.Fn = f32.Fn;
    a.nRK = nRK;
    a.dt = dt;
    a.eleDt = (in.dtType == 2 || perElementDt) ? eleDt : nullptr;
    a.U0 = f32.U0;
    a.acc = f32.acc;
    a.comp = f32.comp;
    a.Uout = f32.U;
    a.err = devErr;
    a.gamma = in.gamma;
    a.ph = ph;
    if (in.viscous) {
      a.dUs = f32.dUs;
      a.dUsStride = (long long)nS * E * nF;
    }
    return a;
  }

  void extrapolate() {
    if (mixed)
      frk::launch_apply_op_t<float>(ext, f32.U, f32.Ufpts, (long long)E * nF, stream);
    else
      frk::launch_apply_op(ext, U, Ufpts, (long long)E * nF, 1.0, 0.0, stream);
    launches++;
    fptsFresh = true;
  }

  // precision form: (U32, comp) from the FP64 boundary copy U, and back
  void split_state() { frk::launch_split((long long)nS * E * nF, U, f32.U, f32.comp, stream); }
  void join_state() { frk::launch_join((long long)nS * E * nF, f32.U, f32.comp, U, stream); }

  // solver::calcDt (solver.cpp:447-468): the first iteration recomputes the
  // wave speeds from U_fpts; afterwards the face kernel's (left-only) values.
  void calc_dt_dev() {
    // coarse P levels never re-initialise (their iteration counter stays at
    // the initial one in the reference, multigrid.cpp:94-98 copies params)
    if (iter == 1 && !pmgCoarse) {
      wavesp_init();
      launches++;
    }
    launches++;
    frk::launch_element_dt_min(nS, nFp, nPF, E, detJ, wSpt, wSurf, waveSp, dA, in.CFL * fr::cfl_limit(in.order),
                               eleDt, dtBits, dtCount, dt, stream);
    // a part on its own rank: the minimum over the ranks (solver.cpp:462-465)
    if (comm && nccl_api().allReduce(dt, dt, 1, ncclDouble, ncclMin, comm, stream) != ncclSuccess) ncclOk = false;
  }

  // Everything of a stage before the element kernel: the common flux Fn (and,
  // viscous, the LDG jumps and the corrected gradients it needs).
  void wavesp_init() {
    if (mo.on)
      frk::launch_wavesp_motion(nDims, nFp, E, Ufpts, norm, mo.a.gVf, in.gamma, waveSp, stream);
    else if (mixed)
      frk::launch_wavesp_init<float>(nDims, nFp, E, f32.Ufpts, norm, in.gamma, waveSp, stream);
    else
      frk::launch_wavesp_init<double>(nDims, nFp, E, Ufpts, norm, in.gamma, waveSp, stream);
  }

  // the face kernels' wave speeds feed only the CFL time step: a batch group
  // (fixed dt per member) does not store them
  double *wave_out() { return perElementDt && in.dtType == 0 ? nullptr : waveSp; }

  void faces_pass() {
    const int nk = (ft.nInterior > 0 ? 1 : 0) + (ft.n > ft.nInterior ? 1 : 0);
    const int nkInv = (nk == 2 && frk::pdl_enabled()) ? 1 : nk;  // small cases: one face launch
    if (mixed) {
      faces_pass32(nk);
      return;
    }
    if (!in.viscous) {
      if (comm && cut.n > 0) exchange_nccl();
      frk::launch_faces_inviscid(nDims, ft, Ufpts, Fn, wave_out(), ph, stream);
      launches += nkInv;
      if (cut.n > 0) {
        frk::launch_faces_cut<double>(nDims, cut, Ufpts, Fn, wave_out(), ph, stream);
        launches++;
      }
      return;
    }
    frk::launch_faces_ldg(nDims, ft, Ufpts, dUc, ph, stream);
    frk::GradArgs g;
    g.E = E;
    g.U = U;
    g.dUc = dUc;
    g.JGinv = JGinv;
    g.detJ = detJ;
    g.dUs = dUs;
    g.dUf = dUf;
    g.sStride = (long long)nS * E * nF;
    g.fStride = (long long)nFp * E * nF;
    if (useTma)
      frk::launch_elem_grad_tma<double>(nDims, in.order, E, tp, tm, devErr, stream);
    else
      frk::launch_elem_grad(nDims, in.order, g, tp, stream);
    frk::launch_faces_visc(nDims, ft, Ufpts, dUf, g.fStride, Fn, wave_out(), ph, stream);
    launches += 2 * nk + 1;
  }
  void faces_pass32(int nk) {
    if (!in.viscous) {
      frk::launch_faces_inviscid<float>(nDims, f32.ft, f32.Ufpts, f32.Fn, wave_out(), ph, stream);
      launches += (nk == 2 && frk::pdl_enabled()) ? 1 : nk;
      return;
    }
    frk::launch_faces_ldg<float>(nDims, f32.ft, f32.Ufpts, f32.dUc, ph, stream);
    frk::GradArgsT<float> g;
    g.E = E;
    g.U = f32.U;
    g.dUc = f32.dUc;
    g.JGinv = f32.JGinv;
    g.detJ = f32.detJ;
    g.dUs = f32.dUs;
    g.dUf = f32.dUf;
    g.sStride = (long long)nS * E * nF;
    g.fStride = (long long)nFp * E * nF;
    if (f32.useTma)
      frk::launch_elem_grad_tma<float>(nDims, in.order, E, f32.tp, f32.tm, devErr, stream);
    else
      frk::launch_elem_grad<float>(nDims, in.order, g, f32.tp, stream);
    frk::launch_faces_visc<float>(nDims, f32.ft, f32.Ufpts, f32.dUf, g.fStride, f32.Fn, wave_out(), ph, stream);
    launches += 2 * nk + 1;
  }
  void element(const frk::ElemArgs &a) {
    if (in.viscous && useTma)
      frk::launch_element_stage_tma_visc<double>(nDims, in.order, a, tp, tm, stream);
    else if (in.viscous)
      frk::launch_element_stage_tp_visc<double>(nDims, in.order, a, tp, stream);
    else if (useTma)
      frk::launch_element_stage_tma<double>(nDims, in.order, a, tp, tm, stream, variant64);
    else if (useTp)
      frk::launch_element_stage_tp<double>(nDims, in.order, a, tp, stream);
    else
      frk::launch_element_stage(nDims, a, stream);
    launches++;
  }
  // precision-form TMA element stage of tile variant v: CUDA-core variants
  // 0 .. tma_variants-1, then the 2-D tensor-core one
  void launch_tma32(const frk::ElemArgsT<float> &a, int v) {
    if (v == frk::tma_variants(true))
      frk::launch_element_stage_tc(nDims, in.order, a, f32.tcOps, f32.tm, stream);
    else
      frk::launch_element_stage_tma<float>(nDims, in.order, a, f32.tp, f32.tm, stream, v);
  }
  void element32(const frk::ElemArgsT<float> &a) {
    if (in.viscous && f32.useTma)
      frk::launch_element_stage_tma_visc<float>(nDims, in.order, a, f32.tp, f32.tm, stream);
    else if (in.viscous)
      frk::launch_element_stage_tp_visc<float>(nDims, in.order, a, f32.tp, stream);
    else if (f32.useTma)
      launch_tma32(a, f32.variant);
    else
      frk::launch_element_stage_tp<float>(nDims, in.order, a, f32.tp, stream);
    launches++;
  }
  // one element-kernel launch of an RK stage in the working precision;
  // divF of the stage is kept when keepDivF (into divF[0])
  frk::ElemArgs stage_args64(int mode, int stage, double rka, double rkb, bool keepDivF, bool pmgSource) {
    frk::ElemArgs a = elem_args();
    a.mode = mode;
    a.stage = stage;
    a.rka_next = rka;
    a.rkb = rkb;
    a.divF_out = keepDivF ? divF[0] : nullptr;
    a.src = pmgSource ? src : nullptr;
    a.Ufpts_out = Ufpts;
    return a;
  }
  frk::ElemArgsT<float> stage_args32(int mode, int stage, double rka, double rkb, bool keepDivF, bool pmgSource) {
    frk::ElemArgsT<float> a = elem_args32();
    a.mode = mode;
    a.stage = stage;
    a.rka_next = rka;
    a.rkb = rkb;
    a.divF_out = keepDivF ? f32.divF[0] : nullptr;
    a.src = pmgSource ? src32 : nullptr;
    a.Ufpts_out = f32.Ufpts;
    return a;
  }
  void element_stage(int mode, int stage, double rka, double rkb, bool keepDivF, bool pmgSource) {
    if (!mixed)
      element(stage_args64(mode, stage, rka, rkb, keepDivF, pmgSource));
    else
      element32(stage_args32(mode, stage, rka, rkb, keepDivF, pmgSource));
  }

  bool calc_residual(int step) {
    if (step < 0 || step >= nRK) return fail(FR_ERR_ARG, "step out of range");
    if (mo.on) {
      residual_motion(step);
      if (Fdbg)
        cudaMemcpyAsync(Fdbg, mo.F, (size_t)nDims * nS * E * nF * sizeof(double), cudaMemcpyDeviceToDevice, stream);
      if (disFnDbg)
        cudaMemcpyAsync(disFnDbg, mo.disFn, (size_t)nFp * E * nF * sizeof(double), cudaMemcpyDeviceToDevice, stream);
      return cuda_ok("calc_residual");
    }
    // the last element stage extrapolated the state it wrote; otherwise
    // (a new or restricted/prolonged state) extrapolate here
    if (!fptsFresh) extrapolate();
    faces_pass();
    if (!mixed) {
      frk::ElemArgs a = elem_args();
      a.mode = frk::MODE_RESIDUAL;
      a.divF_out = divF[step];
      a.F_dbg = Fdbg;
      a.disFn_dbg = disFnDbg;
      element(a);
    } else {
      frk::ElemArgsT<float> a = elem_args32();
      a.mode = frk::MODE_RESIDUAL;
      a.divF_out = f32.divF[step];
      a.F_dbg = f32.Fdbg;
      a.disFn_dbg = f32.disFnDbg;
      element32(a);
    }
    return cuda_ok("calc_residual");
  }

  // solver::update (solver.cpp:319-363)
  bool update_once(bool pmgSource) {
    if (mo.on) return update_motion(pmgSource);
    if (!fptsFresh) extrapolate();
    const bool jameson = in.timeType >= 5;
    for (int step = 0; step < nRK - 1; step++) {
      if (step == 0 && in.dtType != 0) calc_dt_dev();
      faces_pass();
      element_stage(jameson ? frk::MODE_JAMESON : frk::MODE_RK_STAGE, step, in.RKa[step + 1],
                    jameson ? 0.0 : in.RKb[step], step == 0, pmgSource);
    }
    faces_pass();
    if (nRK == 1 && in.dtType != 0) calc_dt_dev();
    if (jameson)
      element_stage(frk::MODE_JAMESON, nRK - 1, in.RKa[nRK], 0.0, nRK == 1, pmgSource);
    else
      element_stage(frk::MODE_RK_FINAL, nRK - 1, 0.0, in.RKb[nRK - 1], nRK == 1, pmgSource);
    // a static coarse P-multigrid level's own time is never read (moving
    // levels advance theirs in update_motion): one launch fewer per coarse
    // step, 12 a driver step at P3 with two smoothing steps
    if (!pmgCoarse) {
      frk::launch_add_time(dt, timeAcc, stream);
      launches++;
    }
    fptsFresh = true;
    return cuda_ok("update");
  }

  bool update(bool pmgSource) {
    if (!stateSet) return fail(FR_ERR_STATE, "no state set");
    iter++;
    return update_once(pmgSource);
  }

  // one step of the driver loop: update, then the P-multigrid cycle when on
  // (reference: flurry.cpp:162-170)
  bool step_once() {
    if (!update_once(false)) return false;
    if (in.PMG && !pmgCoarse && !levels.empty()) return pmg_cycle();
    return true;
  }

  bool run(int n) {
    if (!stateSet) return fail(FR_ERR_STATE, "no state set");
    if (n <= 0) return true;
    // the first iteration differs (wave-speed initialisation); run it eagerly
    while (n > 0 && iter < 1) {
      iter++;
      if (!step_once()) return false;
      n--;
    }
    if (n <= 0) return true;
    // the steady-state step (or kRunChunk of them) captured once
    auto capture = [&](int steps, cudaGraphExec_t &exec, int &kernels) {
      if (!stream) return fail(FR_ERR_STATE, "graph capture needs a non-default stream");
      cudaGraph_t g;
      long long saveIter = iter;
      iter = 2;  // steady-state branch
      if (cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
        return fail(FR_ERR_CUDA, "begin capture");
      long long before = total_launches();
      for (int i = 0; i < steps; i++) step_once();
      kernels = (int)(total_launches() - before);
      launches -= kernels;  // counted again at every replay
      if (cudaStreamEndCapture(stream, &g) != cudaSuccess) return fail(FR_ERR_CUDA, "end capture");
      iter = saveIter;
      if (cudaGraphInstantiate(&exec, g, 0) != cudaSuccess) {
        cudaGraphDestroy(g);
        return fail(FR_ERR_CUDA, "graph instantiate");
      }
      cudaGraphDestroy(g);
      return true;
    };
    if (n >= kRunChunk && !graphK && !capture(kRunChunk, graphK, graphKernelsK)) return false;
    for (; n >= kRunChunk; n -= kRunChunk) {
      iter += kRunChunk;
      if (cudaGraphLaunch(graphK, stream) != cudaSuccess) return fail(FR_ERR_CUDA, "graph launch");
      launches += graphKernelsK;
    }
    if (n > 0 && !graph && !capture(1, graph, graphKernels)) return false;
    for (int i = 0; i < n; i++) {
      iter++;
      if (cudaGraphLaunch(graph, stream) != cudaSuccess) return fail(FR_ERR_CUDA, "graph launch");
      launches += graphKernels;
    }
    return cuda_ok("run");
  }

  bool sync() {
    cudaError_t e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return fail(FR_ERR_CUDA, std::string("sync: ") + cudaGetErrorString(e));
    if (devErr) {
      unsigned int w = 0;
      if (cudaMemcpy(&w, devErr, sizeof(w), cudaMemcpyDeviceToHost) != cudaSuccess)
        return fail(FR_ERR_CUDA, "status read failed");
      if (w) {
        timedOut = true;
        return fail(FR_ERR_TIMEOUT, "a bounded device wait ran out (TMA tile load)");
      }
    }
    if (mo.err) {
      unsigned int w = 0;
      if (cudaMemcpy(&w, mo.err, sizeof(w), cudaMemcpyDeviceToHost) != cudaSuccess)
        return fail(FR_ERR_CUDA, "status read failed");
      if (w) return fail(FR_ERR_SETUP, "Negative Jacobian at solution points.");  // src/solver.cpp:1638
    }
    return true;
  }
  bool timedOut = false;
};

namespace {
// launch policy of a case's calls: PDL on for small cases, restored on exit
struct PdlScope {
  bool prev;
  explicit PdlScope(const fr_case *c) : prev(frk::pdl_enabled()) { frk::set_pdl(c && c->usePdl); }
  ~PdlScope() { frk::set_pdl(prev); }
};
}  // namespace

// Many independent cases advanced together: same-order cases are merged into
// one group case (elements concatenated, faces offset), so each RK stage is
// one face launch and one element launch per order present, and a whole step
// of a group replays as one CUDA graph; groups of different orders run on
// their own streams concurrently.
struct fr_batch {
  std::string err;
  std::vector<fr_case *> members;                 // not owned
  std::vector<std::unique_ptr<fr_case>> groups;   // one per order present
  std::vector<std::vector<int>> groupMembers;     // member indices per group
  std::vector<std::vector<int>> groupOffsets;     // element offset of each member
  long long steps = 0;

  // Many-order form (FR_BATCH_MANY_ORDER): one face launch and one
  // persistent element launch per RK stage for all groups, on one stream
  // (the first group's), a whole step replayed as one CUDA graph.  The
  // merged-group form (FR_BATCH_GROUPS) runs each group's own step graph on
  // its own stream.  fr_batch_create times both and keeps the faster.
  int form = FR_BATCH_GROUPS;
  float formMs[2] = {-1.0f, -1.0f};  // ms per step measured at creation
  unsigned int *ctr = nullptr;        // work counters of the element launch
  std::vector<cudaStream_t> ownStreams;
  cudaGraphExec_t mgraph = nullptr;

  ~fr_batch() {
    if (!groups.empty()) cudaStreamSynchronize(ownStreams.empty() ? groups[0]->stream : ownStreams[0]);
    if (mgraph) cudaGraphExecDestroy(mgraph);
    if (ctr) cudaFree(ctr);
    // the groups own their streams again before they are released
    for (size_t g = 0; g < groups.size() && g < ownStreams.size(); g++) groups[g]->stream = ownStreams[g];
  }

  bool many_order_capable() const {
    if (groups.empty() || (int)groups.size() > frk::kMaxOrderGroups) return false;
    for (auto &g : groups)
      if (!g->useTp || g->in.viscous || g->nDims != groups[0]->nDims || g->mixed != groups[0]->mixed) return false;
    return true;
  }
  void use_streams(bool shared) {
    for (size_t g = 0; g < groups.size(); g++) groups[g]->stream = shared ? ownStreams[0] : ownStreams[g];
  }
  template <typename R>
  void many_faces() {
    frk::MultiFaceArgsT<R> m;
    m.nGroups = (int)groups.size();
    for (int gi = 0; gi < m.nGroups; gi++) {
      fr_case &g = *groups[gi];
      if constexpr (std::is_same<R, double>::value) {
        m.ft[gi] = g.ft;
        m.Uf[gi] = g.Ufpts;
        m.Fn[gi] = g.Fn;
      } else {
        m.ft[gi] = g.f32.ft;
        m.Uf[gi] = g.f32.Ufpts;
        m.Fn[gi] = g.f32.Fn;
      }
      m.wave[gi] = g.wave_out();
      m.istart[gi + 1] = m.istart[gi] + m.ft[gi].nInterior;
      m.bstart[gi + 1] = m.bstart[gi] + (m.ft[gi].n - m.ft[gi].nInterior);
      g.launches++;  // counted once per group: the launch does every group's faces
    }
    frk::launch_faces_multi<R>(groups[0]->nDims, m, groups[0]->ph, ownStreams[0]);
  }
  template <typename R>
  void many_elements(int mode, int stage, double rka, double rkb, bool keepDivF, bool finalStage) {
    frk::MultiElemArgsT<R> m;
    m.nGroups = (int)groups.size();
    for (int gi = 0; gi < m.nGroups; gi++) {
      fr_case &g = *groups[gi];
      if constexpr (std::is_same<R, double>::value) {
        m.a[gi] = g.stage_args64(mode, stage, rka, rkb, keepDivF, false);
        m.t[gi] = g.tp;
      } else {
        m.a[gi] = g.stage_args32(mode, stage, rka, rkb, keepDivF, false);
        m.t[gi] = g.f32.tp;
      }
      m.order[gi] = g.in.order;
      const int eb = frk::tp_elems_per_block<R>(g.nDims, g.in.order);
      m.start[gi + 1] = m.start[gi] + (g.E + eb - 1) / eb;
      m.timeAcc[gi] = g.timeAcc;
      g.launches++;
    }
    m.total = m.start[m.nGroups];
    m.next = ctr;
    m.done = ctr + 1;
    m.finalStage = finalStage ? 1 : 0;
    frk::launch_element_stage_multi<R>(groups[0]->nDims, m, ownStreams[0]);
  }
  // solver::update (src/solver.cpp:319-363) for every group at once
  template <typename R>
  void many_step() {
    fr_case &g0 = *groups[0];
    const int nRK = g0.nRK;
    const bool jameson = g0.in.timeType >= 5;
    for (auto &g : groups)
      if (!g->fptsFresh) g->extrapolate();
    for (int st = 0; st < nRK - 1; st++) {
      many_faces<R>();
      many_elements<R>(jameson ? frk::MODE_JAMESON : frk::MODE_RK_STAGE, st, g0.in.RKa[st + 1],
                       jameson ? 0.0 : g0.in.RKb[st], st == 0, false);
    }
    many_faces<R>();
    if (jameson)
      many_elements<R>(frk::MODE_JAMESON, nRK - 1, g0.in.RKa[nRK], 0.0, nRK == 1, true);
    else
      many_elements<R>(frk::MODE_RK_FINAL, nRK - 1, 0.0, g0.in.RKb[nRK - 1], nRK == 1, true);
    for (auto &g : groups) g->fptsFresh = true;
  }
  bool many_run(int n) {
    if (n <= 0) return true;
    for (auto &g : groups)
      if (!g->sync()) return fail(g->err);
    use_streams(true);
    const bool f32 = groups[0]->mixed;
    // a step with no stale traces is the steady one: capture it once
    for (auto &g : groups)
      if (!g->fptsFresh) {
        f32 ? many_step<float>() : many_step<double>();
        for (auto &h : groups) h->iter++;
        n--;
        break;
      }
    bool ok = true;
    if (n > 0 && !mgraph) {
      cudaGraph_t gr;
      std::vector<long long> l0;
      for (auto &g : groups) l0.push_back(g->launches);
      if (cudaStreamBeginCapture(ownStreams[0], cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        use_streams(false);
        return fail("begin capture");
      }
      f32 ? many_step<float>() : many_step<double>();
      for (size_t i = 0; i < groups.size(); i++) {
        graphLaunches.push_back(groups[i]->launches - l0[i]);
        groups[i]->launches = l0[i];
      }
      if (cudaStreamEndCapture(ownStreams[0], &gr) != cudaSuccess) ok = fail("end capture");
      if (ok && cudaGraphInstantiate(&mgraph, gr, 0) != cudaSuccess) ok = fail("graph instantiate");
      if (ok) cudaGraphDestroy(gr);
    }
    for (int i = 0; ok && i < n; i++) {
      if (cudaGraphLaunch(mgraph, ownStreams[0]) != cudaSuccess) ok = fail("graph launch");
      for (size_t gi = 0; gi < groups.size(); gi++) {
        groups[gi]->iter++;
        groups[gi]->launches += graphLaunches[gi];
      }
    }
    use_streams(false);
    if (ok) {
      const cudaError_t e = cudaGetLastError();
      if (e != cudaSuccess) ok = fail(std::string("many-order step: ") + cudaGetErrorString(e));
    }
    // every group's own stream waits for the steps issued on the first one
    cudaEvent_t ev;
    if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) return fail("event");
    cudaEventRecord(ev, ownStreams[0]);
    for (size_t i = 1; i < ownStreams.size(); i++) cudaStreamWaitEvent(ownStreams[i], ev, 0);
    cudaEventDestroy(ev);
    return ok;
  }
  std::vector<long long> graphLaunches;
  bool groups_run(int n) {
    for (auto &g : groups) {
      PdlScope pdlScope(g.get());
      if (!g->run(n)) return fail(g->err);
    }
    return true;
  }
  bool run(int n) { return form == FR_BATCH_MANY_ORDER ? many_run(n) : groups_run(n); }
  bool fail(const std::string &m) {
    err = m;
    return false;
  }

  // Times `steps` steps of each form on the batch's own state and keeps the
  // faster; the state and time are restored afterwards, so the choice
  // changes the speed only.
  bool autotune_form(int steps) {
    if (!many_order_capable()) return true;
    struct Saved {
      void *U = nullptr, *C = nullptr;
      double t = 0.0;
      long long iter = 0;
    };
    std::vector<Saved> sv(groups.size());
    auto bytesU = [&](fr_case &g) { return (size_t)g.nS * g.E * g.nF * (g.mixed ? sizeof(float) : sizeof(double)); };
    bool ok = true;
    for (size_t i = 0; ok && i < groups.size(); i++) {
      fr_case &g = *groups[i];
      if (!g.sync() || cudaMalloc(&sv[i].U, bytesU(g)) != cudaSuccess ||
          (g.mixed && cudaMalloc(&sv[i].C, bytesU(g)) != cudaSuccess)) {
        ok = fail("autotune: state copy");
        break;
      }
      cudaMemcpy(sv[i].U, g.mixed ? (void *)g.f32.U : (void *)g.U, bytesU(g), cudaMemcpyDeviceToDevice);
      if (g.mixed) cudaMemcpy(sv[i].C, g.f32.comp, bytesU(g), cudaMemcpyDeviceToDevice);
      cudaMemcpy(&sv[i].t, g.timeAcc, sizeof(double), cudaMemcpyDeviceToHost);
      sv[i].iter = g.iter;
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (ok && (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)) ok = fail("events");
    for (int f = 0; ok && f < 2; f++) {
      form = f;
      if (!run(1)) {
        ok = false;
        break;
      }
      for (auto &g : groups) g->sync();
      cudaEventRecord(e0, ownStreams[0]);
      // the groups' own streams join the first one, so e1 closes every group's steps
      for (size_t i = 1; i < groups.size(); i++) cudaStreamWaitEvent(ownStreams[i], e0, 0);
      if (!run(steps)) {
        ok = false;
        break;
      }
      for (size_t i = 1; i < groups.size(); i++) {
        cudaEvent_t ev;
        cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
        cudaEventRecord(ev, ownStreams[i]);
        cudaStreamWaitEvent(ownStreams[0], ev, 0);
        cudaEventDestroy(ev);
      }
      cudaEventRecord(e1, ownStreams[0]);
      if (cudaEventSynchronize(e1) != cudaSuccess) {
        ok = fail("autotune: sync");
        break;
      }
      float ms = 0.0f;
      cudaEventElapsedTime(&ms, e0, e1);
      formMs[f] = ms / steps;
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    form = (ok && formMs[1] > 0.0f && formMs[1] < formMs[0]) ? FR_BATCH_MANY_ORDER : FR_BATCH_GROUPS;
    for (size_t i = 0; i < groups.size(); i++) {
      fr_case &g = *groups[i];
      if (sv[i].U) {
        g.sync();
        cudaMemcpy(g.mixed ? (void *)g.f32.U : (void *)g.U, sv[i].U, bytesU(g), cudaMemcpyDeviceToDevice);
        if (g.mixed) cudaMemcpy(g.f32.comp, sv[i].C, bytesU(g), cudaMemcpyDeviceToDevice);
        cudaMemcpy(g.timeAcc, &sv[i].t, sizeof(double), cudaMemcpyHostToDevice);
        g.iter = sv[i].iter;
        g.fptsFresh = false;
      }
      cudaFree(sv[i].U);
      cudaFree(sv[i].C);
    }
    return ok;
  }
};

// One case split into parts by a partition of its elements, all parts on
// one device and one stream, exchanging the traces of the faces the
// partition cuts through device buffers at every stage: the stepping of the
// reference's MPI runs (mpiFace::communicate / getRightState,
// src/mpiFace.cpp:122-175; the dt MPI_Allreduce, src/solver.cpp:462-465)
// with device-to-device copies in place of the messages.
struct fr_shard {
  std::string err;
  std::unique_ptr<fr_case> full;  // host-side setup of the whole case
  std::vector<int> part;          // part of every element
  std::vector<std::vector<int>> owned;
  std::vector<std::unique_ptr<fr_case>> parts;
  struct Copy {
    int dst, src;
    long long dOff, sOff, n;  // in cut points
  };
  std::vector<Copy> copies;
  std::vector<double *> dts;
  cudaStream_t stream = nullptr;
  cudaGraphExec_t graph = nullptr;
  long long iter = 0;
  bool stateSet = false;

  ~fr_shard() {
    if (stream) cudaStreamSynchronize(stream);
    if (graph) cudaGraphExecDestroy(graph);
    parts.clear();
    if (stream) cudaStreamDestroy(stream);
  }
  bool fail(const std::string &m) {
    err = m;
    return false;
  }

  // the traces of every part's cut points into its send buffer, then each
  // part's receive segment from each peer copied from that peer's send segment
  void exchange() {
    for (auto &p : parts)
      if (p->cut.n > 0) {
        frk::launch_pack_cut<double>(p->nF, p->cut, p->Ufpts, stream);
        p->launches++;
      }
    const int nF = parts[0]->nF;
    for (const Copy &c : copies)
      cudaMemcpyAsync(parts[c.dst]->cut.recv + c.dOff * nF, parts[c.src]->cut.send + c.sOff * nF,
                      (size_t)c.n * nF * sizeof(double), cudaMemcpyDeviceToDevice, stream);
  }
  void global_dt() {
    for (auto &p : parts) p->calc_dt_dev();
    frk::launch_min_dt(dts.data(), (int)dts.size(), stream);
  }
  bool residual(int step) {
    for (auto &p : parts)
      if (!p->fptsFresh) p->extrapolate();
    exchange();
    for (auto &p : parts) {
      p->faces_pass();
      frk::ElemArgs a = p->elem_args();
      a.mode = frk::MODE_RESIDUAL;
      a.divF_out = p->divF[step];
      p->element(a);
    }
    for (auto &p : parts)
      if (!p->cuda_ok("shard residual")) return fail(p->err);
    return true;
  }
  // solver::update (src/solver.cpp:319-363) over all parts, stage by stage
  bool step_once() {
    fr_case &p0 = *parts[0];
    const int nRK = p0.nRK;
    const bool jameson = p0.in.timeType >= 5;
    for (auto &p : parts)
      if (!p->fptsFresh) p->extrapolate();
    for (int st = 0; st < nRK - 1; st++) {
      if (st == 0 && p0.in.dtType != 0) global_dt();
      exchange();
      for (auto &p : parts) {
        p->faces_pass();
        p->element_stage(jameson ? frk::MODE_JAMESON : frk::MODE_RK_STAGE, st, p->in.RKa[st + 1],
                         jameson ? 0.0 : p->in.RKb[st], st == 0, false);
      }
    }
    exchange();
    for (auto &p : parts) p->faces_pass();
    if (nRK == 1 && p0.in.dtType != 0) global_dt();
    for (auto &p : parts) {
      if (jameson)
        p->element_stage(frk::MODE_JAMESON, nRK - 1, p->in.RKa[nRK], 0.0, nRK == 1, false);
      else
        p->element_stage(frk::MODE_RK_FINAL, nRK - 1, 0.0, p->in.RKb[nRK - 1], nRK == 1, false);
      frk::launch_add_time(p->dt, p->timeAcc, stream);
      p->launches++;
      p->fptsFresh = true;
    }
    return true;
  }
  void set_iter(long long it) {
    iter = it;
    for (auto &p : parts) p->iter = it;
  }
  // n driver steps; after the first (which initialises the wave speeds) the
  // step of every part is replayed from one CUDA graph
  bool run(int n) {
    while (n > 0 && iter < 1) {
      set_iter(iter + 1);
      if (!step_once()) return false;
      n--;
    }
    if (n <= 0) return sync();
    if (!graph) {
      cudaGraph_t g;
      const long long save = iter;
      set_iter(2);  // steady-state branch
      if (cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
        return fail("begin capture");
      step_once();
      if (cudaStreamEndCapture(stream, &g) != cudaSuccess) return fail("end capture");
      set_iter(save);
      if (cudaGraphInstantiate(&graph, g, 0) != cudaSuccess) {
        cudaGraphDestroy(g);
        return fail("graph instantiate");
      }
      cudaGraphDestroy(g);
    }
    for (int i = 0; i < n; i++) {
      set_iter(iter + 1);
      if (cudaGraphLaunch(graph, stream) != cudaSuccess) return fail("graph launch");
    }
    return sync();
  }
  bool sync() {
    for (auto &p : parts)
      if (!p->sync()) return fail(p->err);
    return true;
  }
};

namespace {

int status_of(fr_case *c, bool ok, int code = FR_ERR_CUDA) {
  if (ok) return FR_OK;
  if (c->err.find("cudaMalloc") != std::string::npos) return FR_ERR_CUDA;
  return code;
}

int create_common(const char *deck, const fr_mesh *mesh, const fr_setup_opts *opts, fr_case **out) {
  if (!deck || !out) return FR_ERR_ARG;
  *out = nullptr;
  std::unique_ptr<fr_case> c(new fr_case());
  fr_setup_opts o;
  if (opts)
    o = *opts;
  else
    fr_setup_opts_default(&o);
  std::string e;
  if (!fr::read_deck(deck, c->in, e)) {
    c->err = e;
    *out = c.release();
    return e.find("open") != std::string::npos ? FR_ERR_ARG : FR_ERR_UNSUPPORTED;
  }
  if (mesh) {
    if (mesh->nDims != c->in.nDims || !fr::shape_supported(mesh->nDims, mesh->nNodes) || mesh->nEles <= 0 ||
        !mesh->xv || !mesh->c2v) {
      c->err = "mesh does not match the deck (nDims / nNodes) or is empty";
      *out = c.release();
      return FR_ERR_ARG;
    }
    fr::Mesh &m = c->mesh;
    m.nDims = mesh->nDims;
    m.nVerts = mesh->nVerts;
    m.xv.assign(mesh->xv, mesh->xv + (size_t)mesh->nVerts * mesh->nDims);
    m.nEles = mesh->nEles;
    m.nNodes = mesh->nNodes;
    m.c2v.assign(mesh->c2v, mesh->c2v + (size_t)mesh->nEles * mesh->nNodes);
    for (int i = 0; i < mesh->nBndFaces; i++) {
      const int *v = &mesh->bndFaceVerts[(size_t)4 * i];
      m.bndFaceVerts.push_back({v[0], v[1], mesh->nDims == 2 ? -1 : v[2], mesh->nDims == 2 ? -1 : v[3]});
      m.bndFaceBc.push_back(mesh->bndFaceBc[i]);
    }
    for (int d = 0; d < 3; d++) m.period[d] = mesh->period[d];
    m.periodicTol = c->in.periodicTol;
  } else {
    if (c->in.meshType == 0) {
      // mesh file named in the deck, relative to the deck's directory first
      std::string mf = c->in.meshFileName;
      std::string dk = deck;
      size_t sl = dk.find_last_of('/');
      if (!mf.empty() && mf[0] != '/' && sl != std::string::npos) {
        std::string cand = dk.substr(0, sl + 1) + mf;
        if (FILE *fp = std::fopen(cand.c_str(), "r")) {
          std::fclose(fp);
          mf = cand;
        }
      }
      if (!fr::read_gmsh(mf, c->in, c->mesh, e)) {
        c->err = e;
        *out = c.release();
        return e.find("open") != std::string::npos ? FR_ERR_ARG
                                                   : (e.find("not on the B200") != std::string::npos ? FR_ERR_UNSUPPORTED
                                                                                                     : FR_ERR_SETUP);
      }
      std::string e2;
      if (!fr::finalize_input(c->in, e2)) {
        c->err = e2;
        *out = c.release();
        return FR_ERR_UNSUPPORTED;
      }
    } else if (c->in.meshType != 1) {
      c->err = "meshType 2 (overset) is not on the B200 path";
      *out = c.release();
      return FR_ERR_UNSUPPORTED;
    } else if (!fr::create_cartesian_mesh(c->in, c->mesh, e)) {
      c->err = e;
      *out = c.release();
      return FR_ERR_SETUP;
    }
    if (o.perturb && c->in.meshType == 1) fr::perturb_interior_vertices(c->in, c->mesh, o.seed, o.perturb_frac);
  }
  bool ok = c->setup(o);
  int st = FR_OK;
  if (!ok) {
    st = c->errCode == FR_ERR_UNSUPPORTED || c->errCode == FR_ERR_CUDA || c->errCode == FR_ERR_SETUP ||
                 c->errCode == FR_ERR_ARG
             ? c->errCode
             : (c->err.find("cuda") != std::string::npos ? FR_ERR_CUDA : FR_ERR_SETUP);
  }
  *out = c.release();
  return st;
}

template <typename T>
int copy_out(fr_case *c, const std::vector<T> &h, void *host, size_t *count) {
  if (!count) return FR_ERR_ARG;
  size_t cap = *count;
  *count = h.size();
  if (!host) return FR_OK;
  if (cap < h.size()) return FR_ERR_ARG;
  std::memcpy(host, h.data(), h.size() * sizeof(T));
  (void)c;
  return FR_OK;
}

// Copies a device array out as FP64 (FP32 arrays of the precision form are
// widened on the host).
template <typename T>
int copy_dev(fr_case *c, const T *d, size_t n, void *host, size_t *count) {
  if (!count) return FR_ERR_ARG;
  if (!d) {
    c->err = "array not kept (enable debug_arrays)";
    return FR_ERR_STATE;
  }
  size_t cap = *count;
  *count = n;
  if (!host) return FR_OK;
  if (cap < n) return FR_ERR_ARG;
  std::vector<T> tmp;
  void *dst = host;
  if (!std::is_same<T, double>::value) {
    tmp.resize(n);
    dst = tmp.data();
  }
  // on the case's stream, after the work that produced the array
  if (cudaMemcpyAsync(dst, d, n * sizeof(T), cudaMemcpyDeviceToHost, c->stream) != cudaSuccess) {
    c->err = "cudaMemcpy D2H failed";
    return FR_ERR_CUDA;
  }
  if (!c->sync()) return FR_ERR_CUDA;
  if (!std::is_same<T, double>::value)
    for (size_t i = 0; i < n; i++) static_cast<double *>(host)[i] = (double)tmp[i];
  return FR_OK;
}

}  // namespace

extern "C" {

void fr_setup_opts_default(fr_setup_opts *o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->precision = FR_PREC_FP64;
  o->visc_flux_quirk = 1;
  o->tile_variant = -1;
}

int fr_create_from_deck(const char *deck_path, const fr_setup_opts *opts, fr_case **out) {
  return create_common(deck_path, nullptr, opts, out);
}

int fr_create_with_mesh(const char *deck_path, const fr_mesh *mesh, const fr_setup_opts *opts,
                        fr_case **out) {
  if (!mesh) return FR_ERR_ARG;
  return create_common(deck_path, mesh, opts, out);
}

void fr_destroy(fr_case *c) { delete c; }

const char *fr_last_error(const fr_case *c) { return c ? c->err.c_str() : "null case"; }

int fr_get_info(fr_case *c, fr_info *info) {
  if (!c || !info) return FR_ERR_ARG;
  std::memset(info, 0, sizeof(*info));
  info->nDims = c->nDims;
  info->nFields = c->nF;
  info->order = c->in.order;
  info->nEles = c->E;
  info->nSpts = c->nS;
  info->nFpts = c->nFp;
  info->nFaces = (int)c->faces.size();
  info->nFacePts = c->ft.n;
  info->nRKSteps = c->nRK;
  info->precision = c->opts.precision;
  info->dtType = c->in.dtType;
  info->timeType = c->in.timeType;
  info->iter = c->iter;
  info->launches = c->total_launches();
  info->tensor_kernels = (c->mixed ? c->f32.useTma : c->useTma) ? 2 : (c->useTp ? 1 : 0);
  info->tile_variant = c->mixed ? (c->f32.useTma ? c->f32.variant : -1) : (c->useTma ? c->variant64 : -1);
  info->elems_per_block = c->EB;
  if (c->U && !c->hostOnly) {
    if (!c->sync()) return FR_ERR_CUDA;
    cudaMemcpy(&info->time, c->timeAcc, sizeof(double), cudaMemcpyDeviceToHost);
    cudaMemcpy(&info->dt, c->dt, sizeof(double), cudaMemcpyDeviceToHost);
  }
  return FR_OK;
}

int fr_set_stream(fr_case *c, void *stream) {
  if (!c) return FR_ERR_ARG;
  if (c->graph) {
    cudaGraphExecDestroy(c->graph);
    c->graph = nullptr;
  }
  if (c->graphK) {
    cudaGraphExecDestroy(c->graphK);
    c->graphK = nullptr;
  }
  c->stream = (cudaStream_t)stream;
  // the coarse P-multigrid levels run on the case's stream too (left on the
  // old one, a captured step would miss their work)
  for (auto &L : c->levels)
    if (L) L->stream = c->stream;
  return FR_OK;
}

int fr_init_solution(fr_case *c, int kind, const double *prm, int nprm) {
  PdlScope pdlScope(c);
  if (!c) return FR_ERR_ARG;
  if (!c->U) {
    c->err = "host-only case: no device state";
    return FR_ERR_STATE;
  }
  // solver::initializeSolution (src/solver.cpp:1896-1899): a restart deck
  // reads its state from the restart file
  if (kind == fr::IC_DECK && c->in.restart) return fr_read_restart(c, nullptr);
  std::vector<double> U;
  std::string e;
  if (!fr::initial_condition(c->in, c->geo, c->nS, c->E, kind, prm, nprm, U, e)) {
    c->err = e;
    return FR_ERR_ARG;
  }
  return fr_set_state(c, U.data(), U.size());
}

int fr_set_state(fr_case *c, const double *U, size_t count) {
  PdlScope pdlScope(c);
  if (!c || !U) return FR_ERR_ARG;
  if (!c->U) {
    c->err = "host-only case: no device state";
    return FR_ERR_STATE;
  }
  if (count != (size_t)c->nS * c->E * c->nF) {
    c->err = "state size mismatch";
    return FR_ERR_ARG;
  }
  if (cudaMemcpyAsync(c->U, U, count * sizeof(double), cudaMemcpyHostToDevice, c->stream) != cudaSuccess) {
    c->err = "cudaMemcpy H2D failed";
    return FR_ERR_CUDA;
  }
  if (c->mixed) c->split_state();
  c->extrapolate();
  if (c->in.dtType != 0)  // solver::initializeSolution, solver.cpp:1932-1938
    c->wavesp_init();
  c->stateSet = true;
  return c->cuda_ok("set_state") ? FR_OK : FR_ERR_CUDA;
}

int fr_get_state(fr_case *c, double *U, size_t count) {
  PdlScope pdlScope(c);
  if (!c || !U) return FR_ERR_ARG;
  size_t n = (size_t)c->nS * c->E * c->nF;
  if (count != n) {
    c->err = "state size mismatch";
    return FR_ERR_ARG;
  }
  if (c->mixed && c->stateSet) c->join_state();
  return copy_dev(c, c->U, n, U, &count);
}

int fr_get_state_async(fr_case *c, double *U, size_t count) {
  PdlScope pdlScope(c);
  if (!c || !U) return FR_ERR_ARG;
  if (c->hostOnly || !c->stateSet) {
    c->err = c->hostOnly ? "host-only case: no device state" : "no state set";
    return FR_ERR_STATE;
  }
  const size_t n = (size_t)c->nS * c->E * c->nF;
  if (count != n) {
    c->err = "state size mismatch";
    return FR_ERR_ARG;
  }
  if (c->mixed) c->join_state();
  if (cudaMemcpyAsync(U, c->U, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream) != cudaSuccess) {
    cudaGetLastError();
    c->err = "cudaMemcpy D2H failed";
    return FR_ERR_CUDA;
  }
  return FR_OK;
}

int fr_calc_residual(fr_case *c, int step) {
  PdlScope pdlScope(c);
  if (!c) return FR_ERR_ARG;
  if (c->hostOnly) {
    c->err = "host-only case: no device state";
    return FR_ERR_STATE;
  }
  if (!c->stateSet) {
    c->err = "no state set";
    return FR_ERR_STATE;
  }
  return status_of(c, c->calc_residual(step), FR_ERR_ARG);
}

int fr_get_residual(fr_case *c, int step, double *divF, size_t count) {
  if (!c || !divF || step < 0 || step >= c->nRK) return FR_ERR_ARG;
  if (c->hostOnly) {
    c->err = "host-only case: no device state";
    return FR_ERR_STATE;
  }
  size_t n = (size_t)c->nS * c->E * c->nF;
  if (count != n) return FR_ERR_ARG;
  if (c->mixed) return copy_dev(c, c->f32.divF[step], n, divF, &count);
  return copy_dev(c, c->divF[step], n, divF, &count);
}

int fr_update(fr_case *c, int pmg_source) {
  PdlScope pdlScope(c);
  if (!c) return FR_ERR_ARG;
  if (c->hostOnly) {
    c->err = "host-only case: no device state";
    return FR_ERR_STATE;
  }
  if (pmg_source && !c->src) {
    c->err = "no P-multigrid source on this case";
    return FR_ERR_STATE;
  }
  bool ok = c->update(pmg_source != 0);
  return ok ? FR_OK : (c->err == "no state set" ? FR_ERR_STATE : FR_ERR_CUDA);
}

int fr_pmg_cycle(fr_case *c) {
  PdlScope pdlScope(c);
  if (!c) return FR_ERR_ARG;
  if (c->hostOnly || !c->stateSet) {
    c->err = "no device state";
    return FR_ERR_STATE;
  }
  bool ok = c->pmg_cycle();
  return ok ? FR_OK : (c->err.find("no P-multigrid") != std::string::npos ? FR_ERR_STATE : FR_ERR_CUDA);
}

int fr_run(fr_case *c, int nsteps) {
  PdlScope pdlScope(c);
  if (!c || nsteps < 0) return FR_ERR_ARG;
  if (c->hostOnly) {
    c->err = "host-only case: no device state";
    return FR_ERR_STATE;
  }
  bool ok = c->run(nsteps);
  return ok ? FR_OK : (c->err == "no state set" ? FR_ERR_STATE : FR_ERR_CUDA);
}

int fr_calc_dt(fr_case *c, double *dtOut) {
  PdlScope pdlScope(c);
  if (!c) return FR_ERR_ARG;
  if (c->hostOnly) {
    c->err = "host-only case: no device state";
    return FR_ERR_STATE;
  }
  if (!c->stateSet) {
    c->err = "no state set";
    return FR_ERR_STATE;
  }
  if (c->in.CFL <= 0) {
    c->err = "CFL not set";
    return FR_ERR_ARG;
  }
  long long save = c->iter;
  if (c->iter == 0) c->iter = 1;  // wave speeds from the current U_fpts
  if (!c->fptsFresh) c->extrapolate();
  c->calc_dt_dev();
  c->iter = save;
  if (!c->sync()) return FR_ERR_CUDA;
  double d;
  cudaMemcpy(&d, c->dt, sizeof(double), cudaMemcpyDeviceToHost);
  c->hostDt = d;
  if (dtOut) *dtOut = d;
  return FR_OK;
}

int fr_set_dt(fr_case *c, double dt) {
  if (!c || !(dt > 0)) return FR_ERR_ARG;
  if (c->hostOnly) {
    c->err = "host-only case: no device state";
    return FR_ERR_STATE;
  }
  c->hostDt = dt;
  c->in.dt = dt;
  if (cudaMemcpyAsync(c->dt, &c->hostDt, sizeof(double), cudaMemcpyHostToDevice, c->stream) != cudaSuccess)
    return FR_ERR_CUDA;
  return c->sync() ? FR_OK : FR_ERR_CUDA;
}

int fr_residual_norm(fr_case *c, int resType, double *out, int nFields) {
  PdlScope pdlScope(c);
  if (!c || !out || nFields != c->nF || resType < 1 || resType > 3) return FR_ERR_ARG;
  if (c->hostOnly) {
    c->err = "host-only case: no device state";
    return FR_ERR_STATE;
  }
  if (c->mixed)
    frk::launch_residual_norm<float>(c->nS, c->E, c->nF, c->f32.divF[0], c->detJ, c->wSpt, resType, c->eleRes,
                                     c->stream);
  else
    frk::launch_residual_norm<double>(c->nS, c->E, c->nF, c->divF[0], c->detJ, c->wSpt, resType, c->eleRes,
                                      c->stream);
  std::vector<double> er((size_t)c->E * c->nF);
  if (!c->sync()) return FR_ERR_CUDA;
  cudaMemcpy(er.data(), c->eleRes, er.size() * sizeof(double), cudaMemcpyDeviceToHost);
  for (int k = 0; k < c->nF; k++) {
    double r = 0;
    for (int e = 0; e < c->E; e++) {
      double v = er[(size_t)e * c->nF + k];
      if (v != v) {
        c->err = "NaN Encountered in Solution Residual!";
        return FR_ERR_NONFINITE;
      }
      r = resType == 3 ? std::max(r, v) : r + v;
    }
    out[k] = resType == 2 ? std::sqrt(r) : r;
  }
  return FR_OK;
}

int fr_check_state(fr_case *c) {
  PdlScope pdlScope(c);
  if (!c) return FR_ERR_ARG;
  if (c->hostOnly) {
    c->err = "host-only case: no device state";
    return FR_ERR_STATE;
  }
  cudaMemsetAsync(c->bad, 0, sizeof(unsigned), c->stream);
  if (c->mixed)
    frk::launch_check_state<float>(c->nS, c->E, c->nF, c->f32.U, c->bad, c->stream);
  else
    frk::launch_check_state<double>(c->nS, c->E, c->nF, c->U, c->bad, c->stream);
  unsigned b = 0;
  if (!c->sync()) return FR_ERR_CUDA;
  cudaMemcpy(&b, c->bad, sizeof(unsigned), cudaMemcpyDeviceToHost);
  if (b) {
    c->err = "non-finite or non-positive density in the state";
    return FR_ERR_NONFINITE;
  }
  return FR_OK;
}

int fr_get_array(fr_case *c, const char *name, void *host, size_t *count) {
  PdlScope pdlScope(c);
  if (!c || !name || !count) return FR_ERR_ARG;
  std::string n = name;
  size_t nU = (size_t)c->nS * c->E * c->nF, nUf = (size_t)c->nFp * c->E * c->nF;
  if (c->hostOnly && (n == "U_spts" || n == "U0" || n == "U_fpts" || n == "Fn_fpts" || n == "waveSp_fpts" ||
                      n == "dUc_fpts" || n == "dU_spts" || n == "dU_fpts" ||
                      n == "ele_dt" || n == "F_spts" || n == "disFn_fpts" || n.rfind("divF_", 0) == 0)) {
    c->err = "host-only case: no device state";
    return FR_ERR_STATE;
  }
  if (c->mixed) {
    auto &m = c->f32;
    if (n == "U_spts") {
      if (c->stateSet) c->join_state();
      return copy_dev(c, c->U, nU, host, count);
    }
    if (n == "U_comp") return copy_dev(c, m.comp, nU, host, count);
    if (n == "U0") return copy_dev(c, m.U0, nU, host, count);
    if (n == "U_fpts") return copy_dev(c, m.Ufpts, nUf, host, count);
    if (n == "Fn_fpts") return copy_dev(c, m.Fn, nUf, host, count);
    if (n == "F_spts") return copy_dev(c, m.Fdbg, (size_t)c->nDims * nU, host, count);
    if (n == "disFn_fpts") return copy_dev(c, m.disFnDbg, nUf, host, count);
    if (n == "dUc_fpts") return copy_dev(c, m.dUc, nUf, host, count);
    if (n == "dU_spts") return copy_dev(c, m.dUs, (size_t)c->nDims * nU, host, count);
    if (n == "dU_fpts") return copy_dev(c, m.dUf, (size_t)c->nDims * nUf, host, count);
    if (n.rfind("divF_", 0) == 0) {
      int s = std::atoi(n.c_str() + 5);
      if (s < 0 || s >= c->nRK) return FR_ERR_ARG;
      return copy_dev(c, m.divF[s], nU, host, count);
    }
  }
  if (n == "U_spts") return copy_dev(c, c->U, nU, host, count);
  if (n == "U0") return copy_dev(c, c->U0, nU, host, count);
  if (n == "U_fpts") return copy_dev(c, c->Ufpts, nUf, host, count);
  if (n == "Fn_fpts") return copy_dev(c, c->Fn, nUf, host, count);
  if (n == "waveSp_fpts") return copy_dev(c, c->waveSp, (size_t)c->nFp * c->E, host, count);
  if (n == "ele_dt") return copy_dev(c, c->eleDt, (size_t)c->E, host, count);
  if (n == "F_spts") return copy_dev(c, c->Fdbg, (size_t)c->nDims * nU, host, count);
  if (n == "disFn_fpts") return copy_dev(c, c->disFnDbg, nUf, host, count);
  if (n == "dUc_fpts") return copy_dev(c, c->dUc, nUf, host, count);
  if (n == "dU_spts") return copy_dev(c, c->dUs, (size_t)c->nDims * nU, host, count);
  if (n == "dU_fpts") return copy_dev(c, c->dUf, (size_t)c->nDims * nUf, host, count);
  if (n.rfind("divF_", 0) == 0) {
    int s = std::atoi(n.c_str() + 5);
    if (s < 0 || s >= c->nRK) return FR_ERR_ARG;
    return copy_dev(c, c->divF[s], nU, host, count);
  }
  if (n == "tile_ms") {  // precision form: element-stage ms per tile variant timed by the autotuner (-1: not run)
    const std::vector<float> &t = c->mixed ? c->f32.tuneMs : c->tuneMs64;
    std::vector<double> v(t.begin(), t.end());
    return copy_out(c, v, host, count);
  }
  if (n == "pos_spts") return copy_out(c, c->geo.pos_spts, host, count);
  if (n == "detJac_spts") return copy_out(c, c->geo.detJac_spts, host, count);
  if (n == "JGinv_spts") return copy_out(c, c->geo.JGinv_spts, host, count);
  if (n == "norm_fpts") return copy_out(c, c->geo.norm_fpts, host, count);
  if (n == "dA_fpts") return copy_out(c, c->geo.dA_fpts, host, count);
  if (n == "xv") return copy_out(c, c->mesh.xv, host, count);
  if (n == "opp_spts_to_fpts") return copy_out(c, c->op.ext, host, count);
  if (n == "opp_correction") return copy_out(c, c->op.corr, host, count);
  if (n == "opp_prolong") return copy_out(c, c->op.prolong, host, count);
  if (n == "opp_restrict") return copy_out(c, c->op.restrict_, host, count);
  for (int d = 0; d < c->nDims; d++) {
    std::string sd = std::to_string(d);
    if (n == "opp_grad_spts_" + sd) return copy_out(c, c->op.grad[d], host, count);
    if (n == "opp_extrapolateFn_" + sd) return copy_out(c, c->op.extFn[d], host, count);
    if (n == "opp_correctU_" + sd) return copy_out(c, c->op.corrU[d], host, count);
  }
  if (n.rfind("face_", 0) == 0) {
    std::vector<int> v;
    for (auto &f : c->faces) {
      if (n == "face_eL") v.push_back(f.eL);
      else if (n == "face_locL") v.push_back(f.locL);
      else if (n == "face_eR") v.push_back(f.eR);
      else if (n == "face_locR") v.push_back(f.locR);
      else if (n == "face_bc") v.push_back(f.bc);
      else if (n == "face_fptR") {
        for (int j = 0; j < c->nPF; j++) v.push_back(f.eR >= 0 ? f.fptR[j] : -1);
      } else
        return FR_ERR_ARG;
    }
    return copy_out(c, v, host, count);
  }
  c->err = "unknown array " + n;
  return FR_ERR_ARG;
}

int fr_device_ptr(fr_case *c, const char *name, void **ptr, size_t *bytes) {
  if (!c || !name || !ptr) return FR_ERR_ARG;
  if (c->hostOnly) {
    c->err = "host-only case: no device state";
    return FR_ERR_STATE;
  }
  std::string n = name;
  size_t nU = (size_t)c->nS * c->E * c->nF, nUf = (size_t)c->nFp * c->E * c->nF;
  void *p = nullptr;
  size_t b = 0;
  if (c->mixed) {  // the precision form's FP32 working arrays
    if (n == "U_spts") {
      p = c->f32.U;
      b = nU * 4;
    } else if (n == "U_fpts") {
      p = c->f32.Ufpts;
      b = nUf * 4;
    } else if (n == "Fn_fpts") {
      p = c->f32.Fn;
      b = nUf * 4;
    } else if (n.rfind("divF_", 0) == 0) {
      int s = std::atoi(n.c_str() + 5);
      if (s < 0 || s >= c->nRK) return FR_ERR_ARG;
      p = c->f32.divF[s];
      b = nU * 4;
    } else {
      return FR_ERR_ARG;
    }
    *ptr = p;
    if (bytes) *bytes = b;
    return FR_OK;
  }
  if (n == "U_spts") {
    p = c->U;
    b = nU * 8;
  } else if (n == "U_fpts") {
    p = c->Ufpts;
    b = nUf * 8;
  } else if (n == "Fn_fpts") {
    p = c->Fn;
    b = nUf * 8;
  } else if (n.rfind("divF_", 0) == 0) {
    int s = std::atoi(n.c_str() + 5);
    if (s < 0 || s >= c->nRK) return FR_ERR_ARG;
    p = c->divF[s];
    b = nU * 8;
  } else {
    return FR_ERR_ARG;
  }
  *ptr = p;
  if (bytes) *bytes = b;
  return FR_OK;
}

int fr_bench_kernel(fr_case *c, const char *kernel, int reps) {
  PdlScope pdlScope(c);
  if (!c || !kernel || reps < 0) return FR_ERR_ARG;
  if (c->hostOnly || !c->stateSet) {
    c->err = "no device state";
    return FR_ERR_STATE;
  }
  std::string k = kernel;
  if (k == "faces") {
    for (int i = 0; i < reps; i++) c->faces_pass();
  } else if (k == "element_stage") {
    const int mode = c->in.timeType >= 5 ? frk::MODE_JAMESON : frk::MODE_RK_STAGE;
    const int stage = c->nRK > 1 ? 1 : 0;
    const double rka = c->in.RKa.size() > 2 ? c->in.RKa[2] : 0.0;
    const double rkb = c->in.RKb.size() > 1 ? c->in.RKb[1] : 0.0;
    for (int i = 0; i < reps; i++) c->element_stage(mode, stage, rka, rkb, false, false);
  } else {
    c->err = "unknown kernel " + k;
    return FR_ERR_ARG;
  }
  return c->cuda_ok("bench_kernel") ? FR_OK : FR_ERR_CUDA;
}

int fr_batch_create(fr_case *const *cases, int n, fr_batch **out) {
  if (!cases || n <= 0 || !out) return FR_ERR_ARG;
  *out = nullptr;
  std::unique_ptr<fr_batch> b(new fr_batch());
  for (int i = 0; i < n; i++) {
    fr_case *c = cases[i];
    if (!c || c->hostOnly || !c->stateSet) return FR_ERR_STATE;
    if (c->in.viscous || c->in.PMG || c->in.motion || c->in.dtType != 0 || c->in.nDims != cases[0]->in.nDims ||
        c->in.timeType != cases[0]->in.timeType || c->opts.precision != cases[0]->opts.precision) {
      return FR_ERR_UNSUPPORTED;  // batches hold inviscid, static-mesh, fixed-dt cases of one RK scheme and precision
    }
    b->members.push_back(c);
  }
  std::vector<int> orders;
  for (auto *c : b->members)
    if (std::find(orders.begin(), orders.end(), c->in.order) == orders.end()) orders.push_back(c->in.order);
  std::sort(orders.begin(), orders.end());
  for (int P : orders) {
    std::vector<fr_case *> ms;
    std::vector<int> idx, offs;
    int off = 0;
    for (int i = 0; i < n; i++)
      if (b->members[i]->in.order == P) {
        ms.push_back(b->members[i]);
        idx.push_back(i);
        offs.push_back(off);
        off += b->members[i]->E;
      }
    std::unique_ptr<fr_case> g(new fr_case());
    fr_setup_opts o = ms[0]->opts;
    if (!g->merge_from(ms, o)) {
      *out = b.release();
      (*out)->err = g->err;
      return FR_ERR_CUDA;
    }
    b->ownStreams.push_back(g->stream);
    b->groups.push_back(std::move(g));
    b->groupMembers.push_back(idx);
    b->groupOffsets.push_back(offs);
  }
  if (b->many_order_capable()) {
    if (cudaMalloc(&b->ctr, 2 * sizeof(unsigned int)) != cudaSuccess ||
        cudaMemset(b->ctr, 0, 2 * sizeof(unsigned int)) != cudaSuccess) {
      b->err = "work counters";
      *out = b.release();
      return FR_ERR_CUDA;
    }
    if (!b->autotune_form(3)) {
      *out = b.release();
      return FR_ERR_CUDA;
    }
  }
  *out = b.release();
  return FR_OK;
}

int fr_batch_form(fr_batch *b, int *form, float *ms_groups, float *ms_many_order) {
  if (!b) return FR_ERR_ARG;
  if (form) *form = b->form;
  if (ms_groups) *ms_groups = b->formMs[0];
  if (ms_many_order) *ms_many_order = b->formMs[1];
  return FR_OK;
}

int fr_batch_set_form(fr_batch *b, int form) {
  if (!b || (form != FR_BATCH_GROUPS && form != FR_BATCH_MANY_ORDER)) return FR_ERR_ARG;
  if (form == FR_BATCH_MANY_ORDER && !b->many_order_capable()) {
    b->err = "the many-order form needs inviscid tensor-product groups of one precision (at most 6 orders)";
    return FR_ERR_UNSUPPORTED;
  }
  for (auto &g : b->groups)
    if (!g->sync()) return FR_ERR_CUDA;
  b->form = form;
  return FR_OK;
}

int fr_batch_run(fr_batch *b, int nsteps) {
  if (!b || nsteps < 0) return FR_ERR_ARG;
  if (!b->run(nsteps)) return FR_ERR_CUDA;
  for (auto &g : b->groups)
    if (!g->sync()) {
      b->err = g->err;
      return g->timedOut ? FR_ERR_TIMEOUT : FR_ERR_CUDA;
    }
  b->steps += nsteps;
  return FR_OK;
}

int fr_batch_gather(fr_batch *b) {
  if (!b) return FR_ERR_ARG;
  for (size_t gi = 0; gi < b->groups.size(); gi++) {
    fr_case &g = *b->groups[gi];
    for (size_t k = 0; k < b->groupMembers[gi].size(); k++)
      if (!g.scatter_to(*b->members[b->groupMembers[gi][k]], b->groupOffsets[gi][k])) {
        b->err = g.err;
        return FR_ERR_CUDA;
      }
    if (!g.sync()) {
      b->err = g.err;
      return FR_ERR_CUDA;
    }
  }
  return FR_OK;
}

int fr_batch_residual_norms(fr_batch *b, int resType, double *out, int nFields) {
  if (!b || !out || resType < 1 || resType > 3 || b->groups.empty() || nFields != b->groups[0]->nF)
    return FR_ERR_ARG;
  for (size_t gi = 0; gi < b->groups.size(); gi++) {
    fr_case &g = *b->groups[gi];
    if (g.mixed)
      frk::launch_residual_norm<float>(g.nS, g.E, g.nF, g.f32.divF[0], g.detJ, g.wSpt, resType, g.eleRes, g.stream);
    else
      frk::launch_residual_norm<double>(g.nS, g.E, g.nF, g.divF[0], g.detJ, g.wSpt, resType, g.eleRes, g.stream);
    std::vector<double> er((size_t)g.E * g.nF);
    if (!g.sync()) return FR_ERR_CUDA;
    cudaMemcpy(er.data(), g.eleRes, er.size() * sizeof(double), cudaMemcpyDeviceToHost);
    for (size_t k = 0; k < b->groupMembers[gi].size(); k++) {
      const int mi = b->groupMembers[gi][k], e0 = b->groupOffsets[gi][k], Em = b->members[mi]->E;
      for (int f = 0; f < g.nF; f++) {
        double r = 0;
        for (int e = e0; e < e0 + Em; e++) {
          double v = er[(size_t)e * g.nF + f];
          r = resType == 3 ? std::max(r, v) : r + v;
        }
        out[(size_t)mi * nFields + f] = resType == 2 ? std::sqrt(r) : r;
      }
    }
  }
  return FR_OK;
}

int fr_batch_info(fr_batch *b, int *nGroups, long long *launches) {
  if (!b) return FR_ERR_ARG;
  if (nGroups) *nGroups = (int)b->groups.size();
  if (launches) {
    long long n = 0;
    for (auto &g : b->groups) n += g->total_launches();
    *launches = n;
  }
  return FR_OK;
}

const char *fr_batch_last_error(const fr_batch *b) { return b ? b->err.c_str() : "null batch"; }

void fr_batch_destroy(fr_batch *b) { delete b; }

int fr_stream_idle(fr_case *c) {
  if (!c || c->hostOnly || !c->stream) return FR_ERR_ARG;
  const cudaError_t e = cudaStreamQuery(c->stream);
  if (e == cudaSuccess) return 1;
  if (e == cudaErrorNotReady) return 0;
  cudaGetLastError();
  c->err = std::string("stream query: ") + cudaGetErrorString(e);
  return -FR_ERR_CUDA;
}

int fr_checkpoint(fr_case *c) {
  PdlScope pdlScope(c);
  if (!c) return FR_ERR_ARG;
  if (c->hostOnly || !c->stateSet) {
    c->err = c->hostOnly ? "host-only case: no device state" : "no state set";
    return FR_ERR_STATE;
  }
  auto &k = c->cp;
  const int n3 = c->in.order + 3;
  const size_t nV = (size_t)(c->nDims == 2 ? n3 * n3 : n3 * n3 * n3) * c->E * c->nF + 1;
  if (!k.Vp) {
    k.nP = c->nDims == 2 ? n3 * n3 : n3 * n3 * n3;
    if (!c->upload(k.opp, fr::spts_to_ppts(c->nDims, c->in.order, c->in.sptsTypeQuad)) || !c->alloc(k.Vp, nV))
      return FR_ERR_CUDA;
    const size_t nX = c->mo.on ? 2 * (size_t)c->mesh.nVerts * c->nDims : 0;
    if (nX && (!c->alloc(k.xv, nX) || cudaMallocHost(&k.xvHost, nX * sizeof(double)) != cudaSuccess)) {
      cudaGetLastError();
      c->err = "cannot allocate the checkpoint buffers";
      return FR_ERR_CUDA;
    }
    if (cudaMallocHost(&k.host, nV * sizeof(double)) != cudaSuccess ||
        cudaStreamCreateWithFlags(&k.copy, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&k.ready, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&k.done, cudaEventDisableTiming) != cudaSuccess) {
      cudaGetLastError();
      c->err = "cannot allocate the checkpoint buffers";
      return FR_ERR_CUDA;
    }
  }
  // the previous copy must have left Vp before the kernel overwrites it
  if (k.pending) cudaStreamWaitEvent(c->stream, k.done, 0);
  if (c->mixed) c->join_state();
  frk::launch_plot_primitives(c->nDims, c->U, k.opp, k.Vp, c->nS, k.nP, c->E, c->in.gamma, c->stream);
  c->launches++;
  cudaMemcpyAsync(k.Vp + nV - 1, c->timeAcc, sizeof(double), cudaMemcpyDeviceToDevice, c->stream);
  const size_t nX = c->mo.on ? (size_t)c->mesh.nVerts * c->nDims : 0;
  if (nX) {
    cudaMemcpyAsync(k.xv, c->mo.a.xv, nX * sizeof(double), cudaMemcpyDeviceToDevice, c->stream);
    cudaMemcpyAsync(k.xv + nX, c->mo.a.gv, nX * sizeof(double), cudaMemcpyDeviceToDevice, c->stream);
  }
  cudaEventRecord(k.ready, c->stream);
  cudaStreamWaitEvent(k.copy, k.ready, 0);
  cudaMemcpyAsync(k.host, k.Vp, nV * sizeof(double), cudaMemcpyDeviceToHost, k.copy);
  if (nX) cudaMemcpyAsync(k.xvHost, k.xv, 2 * nX * sizeof(double), cudaMemcpyDeviceToHost, k.copy);
  cudaEventRecord(k.done, k.copy);
  k.pending = true;
  k.iter = c->iter;
  return c->cuda_ok("checkpoint") ? FR_OK : FR_ERR_CUDA;
}

int fr_write_data(fr_case *c, const char *path) {
  if (!c) return FR_ERR_ARG;
  if (c->hostOnly || !c->stateSet) {
    c->err = c->hostOnly ? "host-only case: no device state" : "no state set";
    return FR_ERR_STATE;
  }
  std::string e;
  char name[64];
  if (c->in.plotType == 0) {
    // src/output.cpp:60-135: primitives at the solution and flux points
    const size_t nU = (size_t)c->nS * c->E * c->nF, nUf = (size_t)c->nFp * c->E * c->nF;
    std::vector<double> U(nU), Uf(nUf);
    size_t cnt = nU;
    int st = fr_get_array(c, "U_spts", U.data(), &cnt);
    if (st != FR_OK) return st;
    if (!c->fptsFresh) c->extrapolate();
    cnt = nUf;
    if ((st = fr_get_array(c, "U_fpts", Uf.data(), &cnt)) != FR_OK) return st;
    std::snprintf(name, sizeof name, ".csv.%.09lld", c->iter);
    const std::string out = path ? std::string(path) : c->in.dataFileName + name;
    if (!fr::write_csv(out, c->nDims, c->nS, c->nFp, c->E, U.data(), Uf.data(), c->geo.pos_spts.data(),
                       c->geo.pos_fpts.data(), c->in.gamma, e)) {
      c->err = e;
      return FR_ERR_ARG;
    }
    return FR_OK;
  }
  auto &k = c->cp;
  if (!k.pending) {
    const int st = fr_checkpoint(c);
    if (st != FR_OK) return st;
  }
  if (cudaEventSynchronize(k.done) != cudaSuccess) {
    cudaGetLastError();
    c->err = "checkpoint copy failed";
    return FR_ERR_CUDA;
  }
  k.pending = false;
  if (c->mo.on) {  // the vertices (and their velocities) where the snapshot was taken
    const size_t nX = (size_t)c->mesh.nVerts * c->nDims;
    const auto loc = fr::loc_ppts(c->nDims, c->in.order, c->in.sptsTypeQuad);
    fr::Mesh moved = c->mesh;
    std::copy(k.xvHost, k.xvHost + nX, moved.xv.begin());
    k.pos.clear();
    bool ok = fr::positions_at(moved, loc, k.pos, e);
    std::copy(k.xvHost + nX, k.xvHost + 2 * nX, moved.xv.begin());  // velocities interpolate the same way
    ok = ok && fr::positions_at(moved, loc, k.gridVel, e);
    if (!ok) {
      c->err = e;
      return FR_ERR_ARG;
    }
  } else if (k.pos.empty() &&
             !fr::positions_at(c->mesh, fr::loc_ppts(c->nDims, c->in.order, c->in.sptsTypeQuad), k.pos, e)) {
    c->err = e;
    return FR_ERR_ARG;
  }
  std::snprintf(name, sizeof name, "_%.09lld.vtu", k.iter);
  const std::string out = path ? std::string(path) : c->in.dataFileName + name;
  const double time = k.host[(size_t)k.nP * c->E * c->nF];
  if (!fr::write_paraview(out, c->nDims, c->in.order, c->E, time, k.iter, k.host, k.pos.data(),
                          c->mo.on ? k.gridVel.data() : nullptr, e)) {
    c->err = e;
    return FR_ERR_ARG;
  }
  return FR_OK;
}

int fr_read_restart(fr_case *c, const char *path) {
  if (!c) return FR_ERR_ARG;
  if (c->hostOnly) {
    c->err = "host-only case: no device state";
    return FR_ERR_STATE;
  }
  char name[64];
  std::snprintf(name, sizeof name, "_%.09d.vtu", c->in.restartIter);
  const std::string in = path ? std::string(path) : c->in.dataFileName + name;
  std::vector<double> U;
  double time = 0.0;
  long long iter = 0;
  bool hasTime = false, hasIter = false;
  std::string e;
  if (!fr::read_restart_vtu(in, c->in, c->in.order, c->E, U, time, hasTime, iter, hasIter, e)) {
    c->err = e;
    return FR_ERR_ARG;
  }
  int st = fr_set_state(c, U.data(), U.size());
  if (st != FR_OK) return st;
  // src/solver.cpp:1829-1836: the simulation time from the file's comment;
  // the iteration count is the deck's restartIter (src/input.cpp:463-467)
  if (hasTime && cudaMemcpy(c->timeAcc, &time, sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) {
    c->err = "cudaMemcpy H2D failed";
    return FR_ERR_CUDA;
  }
  if (!path) c->iter = c->in.restartIter;
  else if (hasIter) c->iter = iter;
  if (c->mo.on) {  // the mesh at the restart time (src/solver.cpp:1855-1857)
    PdlScope pdlScope(c);
    c->move_mesh(0.0);
    // P-multigrid levels keep their own time, which starts at zero: they copy
    // the inputs before the finest level reads the restart file and reset
    // their time in their own setup (multigrid.cpp:52, 131-136 with
    // solver.cpp:76)
    if (!c->cuda_ok("restart")) return FR_ERR_CUDA;
  }
  return FR_OK;
}

int fr_integrate_error(fr_case *c, int errorNorm, double *out, int nFields) {
  PdlScope pdlScope(c);
  if (!c || !out) return FR_ERR_ARG;
  if (c->hostOnly || !c->stateSet) {
    c->err = c->hostOnly ? "host-only case: no device state" : "no state set";
    return FR_ERR_STATE;
  }
  if (nFields != c->nF) {
    c->err = "nFields mismatch";
    return FR_ERR_ARG;
  }
  const int norm = errorNorm < 0 ? c->in.errorNorm : errorNorm;
  if (norm < 0 || norm > 2) {
    c->err = "errorNorm must be 0, 1 or 2";
    return FR_ERR_ARG;
  }
  const int nd = c->nDims, nN = c->mesh.nNodes;
  // tables: errorNorm 0 on the solution points, 1 and 2 on quadOrder points
  auto &T = c->errT[norm == 0 ? 0 : 1];
  if (!T.opQ) {
    std::vector<fr::Pt> loc;
    std::vector<double> op, w;
    const int n = c->in.order + 1;
    if (norm == 0) {
      loc = fr::loc_spts(nd, c->in.order, c->in.sptsTypeQuad);
      op.assign((size_t)c->nS * c->nS, 0.0);
      for (int s2 = 0; s2 < c->nS; s2++) op[(size_t)s2 * c->nS + s2] = 1.0;
      w = fr::spt_weights(nd, c->in.order);
    } else {
      if (c->in.quadOrder < 0 || c->in.quadOrder > 10) {
        c->err = "quadOrder must be in 0..10";  // the reference's weight tables (src/points.cpp:435-520)
        return FR_ERR_ARG;
      }
      loc = fr::loc_spts(nd, c->in.quadOrder, fr::PTS_LEGENDRE);
      w = fr::spt_weights(nd, c->in.quadOrder);
      const std::vector<double> s1 = fr::pts1d(c->in.sptsTypeQuad, c->in.order);
      op.assign(loc.size() * c->nS, 0.0);
      for (size_t q = 0; q < loc.size(); q++)  // src/operators.cpp:241-280
        for (int s2 = 0; s2 < c->nS; s2++) {
          double v = fr::lagrange(s1, loc[q].x, s2 % n) * fr::lagrange(s1, loc[q].y, (s2 / n) % n);
          if (nd == 3) v *= fr::lagrange(s1, loc[q].z, s2 / (n * n));
          op[q * c->nS + s2] = v;
        }
    }
    std::vector<double> N, dN;
    std::string e;
    if (!fr::shape_tables(nd, nN, loc, N, dN, e)) {
      c->err = e;
      return FR_ERR_ARG;
    }
    if (!c->upload(T.opQ, op) || !c->upload(T.wQ, w) || !c->upload(T.shapeQ, N)) return FR_ERR_CUDA;
    T.nQ = (int)loc.size();
  }
  if (!c->errElem) {
    if (!c->alloc(c->errElem, 2 * (size_t)c->E * c->nF) || !c->alloc(c->errOut, c->nF)) return FR_ERR_CUDA;
    if (!c->mo.on) {
      std::vector<double> xv(c->mesh.xv.begin(), c->mesh.xv.begin() + (size_t)c->mesh.nVerts * nd);
      if (!c->upload(c->errXv, xv) || !c->upload(c->errC2v, c->mesh.c2v)) return FR_ERR_CUDA;
    }
  }
  frk::ErrorArgs a;
  a.nDims = nd;
  a.nS = c->nS;
  a.nQ = T.nQ;
  a.E = c->E;
  a.nF = c->nF;
  a.nNodes = nN;
  a.icType = c->in.icType;
  a.testCase = c->in.testCase;
  a.errorNorm = norm;
  a.gamma = c->in.gamma;
  a.pIC = c->in.pIC;
  a.rhoIC = c->in.rhoIC;
  a.vortexAngle = c->in.vortexAngle;
  a.pi = 4.0 * std::atan(1.0);  // the reference's pi (include/global.hpp:72)
  // periodic box of the exact vortex (src/funcs.cpp:1349-1358, 1391-1400)
  if (c->in.meshType == 1) {
    a.xmin = c->in.xmin, a.xmax = c->in.xmax, a.ymin = c->in.ymin, a.ymax = c->in.ymax;
  } else if (c->in.icType == 2) {
    a.xmin = c->in.vortexXmin, a.xmax = c->in.vortexXmax, a.ymin = c->in.vortexYmin, a.ymax = c->in.vortexYmax;
  }
  a.time = c->timeAcc;
  if (c->mixed) c->join_state();
  a.U = c->U;
  a.detJ = c->detJ;
  a.opQ = T.opQ;
  a.wQ = T.wQ;
  a.shapeQ = T.shapeQ;
  a.xv = c->mo.on ? c->mo.a.xv : c->errXv;
  a.c2v = c->mo.on ? c->mo.a.c2v : c->errC2v;
  a.elemErr = c->errElem;
  a.elemU = c->errElem + (size_t)c->E * c->nF;
  frk::launch_error_integral(a, c->errOut, c->stream);
  c->launches += 2;
  if (cudaMemcpyAsync(out, c->errOut, c->nF * sizeof(double), cudaMemcpyDeviceToHost, c->stream) != cudaSuccess) {
    cudaGetLastError();
    c->err = "cudaMemcpy D2H failed";
    return FR_ERR_CUDA;
  }
  return c->sync() ? FR_OK : FR_ERR_CUDA;
}

int fr_wall_force(fr_case *c, double *out) {
  PdlScope pdlScope(c);
  if (!c || !out) return FR_ERR_ARG;
  if (c->hostOnly || !c->stateSet) {
    c->err = c->hostOnly ? "host-only case: no device state" : "no state set";
    return FR_ERR_STATE;
  }
  double v[11];
  if (!c->boundary_monitors(0, v)) return FR_ERR_CUDA;
  // writeResidual (src/output.cpp:1048-1066): coefficients on 0.5 rho U^2 of
  // the boundary state, turned to the free-stream direction
  const auto &in = c->in;
  const double wB = c->nDims == 2 ? 0.0 : in.wBound;
  const double Uinf = std::sqrt(in.uBound * in.uBound + in.vBound * in.vBound + wB * wB);
  double f[6];
  for (int k = 0; k < 6; k++) f[k] = v[k] / (0.5 * in.rhoBound * Uinf * Uinf);
  const double alpha = std::atan2(in.vBound, in.uBound);
  out[0] = f[0] * std::cos(alpha) + f[1] * std::sin(alpha);
  out[1] = f[1] * std::cos(alpha) - f[0] * std::sin(alpha);
  out[2] = f[2];
  out[3] = in.viscous ? f[3] * std::cos(alpha) + f[4] * std::sin(alpha) : f[3];
  out[4] = in.viscous ? f[4] * std::cos(alpha) - f[3] * std::sin(alpha) : f[4];
  out[5] = f[5];
  return FR_OK;
}

int fr_mass_flux(fr_case *c, int errorNorm, double *out, int nFields) {
  PdlScope pdlScope(c);
  if (!c || !out) return FR_ERR_ARG;
  if (c->hostOnly || !c->stateSet) {
    c->err = c->hostOnly ? "host-only case: no device state" : "no state set";
    return FR_ERR_STATE;
  }
  const int norm = errorNorm < 0 ? c->in.errorNorm : errorNorm;
  if (nFields != c->nF || norm < 0 || norm > 2) {
    c->err = "nFields mismatch or errorNorm outside 0..2";
    return FR_ERR_ARG;
  }
  double v[11];
  if (!c->boundary_monitors(norm, v)) return FR_ERR_CUDA;
  for (int k = 0; k < c->nF; k++) out[k] = v[6 + k];
  return FR_OK;
}

int fr_shard_plan(fr_case *c, int nparts, int rank, int *part, int *n_owned, long long *n_halo, int *halo_peer,
                  long long *halo_slot, long long cap) {
  if (!c || !n_owned || !n_halo || nparts < 1 || rank < 0 || rank >= nparts || cap < 0) return FR_ERR_ARG;
  if (cap > 0 && (!halo_peer || !halo_slot)) return FR_ERR_ARG;
  if (c->in.motion != 0) {
    c->err = "sharding plan: moving meshes are not partitioned";
    return FR_ERR_UNSUPPORTED;
  }
  std::vector<int> pt, owned, peer;
  std::vector<long long> slot;
  if (!fr::partition_elements(c->mesh, nparts, pt, c->err) ||
      !fr::halo_plan(c->mesh, c->faces, c->nPF, pt, rank, owned, peer, slot, c->err))
    return FR_ERR_ARG;
  if (part) std::copy(pt.begin(), pt.end(), part);
  *n_owned = (int)owned.size();
  *n_halo = (long long)slot.size();
  if (cap > 0) {
    if (cap < (long long)slot.size()) {
      c->err = "sharding plan: halo buffers smaller than the halo";
      return FR_ERR_ARG;
    }
    std::copy(peer.begin(), peer.end(), halo_peer);
    std::copy(slot.begin(), slot.end(), halo_slot);
  }
  return FR_OK;
}

int fr_shard_create(const char *deck_path, const fr_setup_opts *opts, int nparts, fr_shard **out) {
  if (!deck_path || !out || nparts < 1 || nparts > frk::kMaxParts) return FR_ERR_ARG;
  *out = nullptr;
  fr_setup_opts o;
  if (opts)
    o = *opts;
  else
    fr_setup_opts_default(&o);
  const int device = o.device;
  if (device < 0) return FR_ERR_ARG;
  std::unique_ptr<fr_shard> sh(new fr_shard());
  fr_setup_opts ho = o;
  ho.device = -1;  // the whole case on the host only: mesh, faces, metrics, operators
  fr_case *f = nullptr;
  int st = create_common(deck_path, nullptr, &ho, &f);
  sh->full.reset(f);
  if (st != FR_OK) {
    sh->err = f ? f->err : "setup failed";
    *out = sh.release();
    return st;
  }
  fr_case &F = *sh->full;
  if (o.precision != FR_PREC_FP64 || F.in.viscous || F.in.PMG || F.in.motion) {
    sh->err = "sharded cases: plain form (FP64), inviscid, static mesh, no P-multigrid";
    *out = sh.release();
    return FR_ERR_UNSUPPORTED;
  }
  if (nparts > F.E || !fr::partition_elements(F.mesh, nparts, sh->part, sh->err)) {
    if (sh->err.empty()) sh->err = "more parts than elements";
    *out = sh.release();
    return FR_ERR_ARG;
  }
  if (cudaSetDevice(device) != cudaSuccess ||
      cudaStreamCreateWithFlags(&sh->stream, cudaStreamNonBlocking) != cudaSuccess) {
    sh->err = "stream create";
    *out = sh.release();
    return FR_ERR_CUDA;
  }
  sh->owned.assign(nparts, {});
  for (int e = 0; e < F.E; e++) sh->owned[sh->part[e]].push_back(e);
  for (int r = 0; r < nparts; r++) {
    std::unique_ptr<fr_case> p(new fr_case());
    if (!p->split_from(F, sh->part, r, sh->stream)) {
      sh->err = "part " + std::to_string(r) + ": " + p->err;
      *out = sh.release();
      return FR_ERR_CUDA;
    }
    sh->dts.push_back(p->dt);
    sh->parts.push_back(std::move(p));
  }
  // copies: part r's segment from peer q <- q's segment for r (same length)
  auto segment = [&](int r, int q, long long &off, long long &n) {
    const auto &cp = sh->parts[r]->cutPeer;
    auto lo = std::lower_bound(cp.begin(), cp.end(), q), hi = std::upper_bound(cp.begin(), cp.end(), q);
    off = lo - cp.begin();
    n = hi - lo;
  };
  for (int r = 0; r < nparts; r++)
    for (int q = 0; q < nparts; q++) {
      if (q == r) continue;
      long long dOff, n1, sOff, n2;
      segment(r, q, dOff, n1);
      segment(q, r, sOff, n2);
      if (n1 != n2) {
        sh->err = "cut lists of two parts disagree";
        *out = sh.release();
        return FR_ERR_SETUP;
      }
      if (n1 > 0) sh->copies.push_back({r, q, dOff, sOff, n1});
    }
  *out = sh.release();
  return FR_OK;
}

int fr_part_create(const char *deck_path, const fr_setup_opts *opts, int nparts, int rank, void *nccl_comm,
                   fr_case **out) {
  if (!deck_path || !out || nparts < 1 || rank < 0 || rank >= nparts || (nparts > 1 && !nccl_comm))
    return FR_ERR_ARG;
  *out = nullptr;
  fr_setup_opts o;
  if (opts)
    o = *opts;
  else
    fr_setup_opts_default(&o);
  if (o.device < 0) return FR_ERR_ARG;
  fr_setup_opts ho = o;
  ho.device = -1;
  fr_case *f = nullptr;
  int st = create_common(deck_path, nullptr, &ho, &f);
  std::unique_ptr<fr_case> full(f);
  std::unique_ptr<fr_case> p(new fr_case());
  auto give = [&](int code, const std::string &m) {
    p->err = m;
    *out = p.release();
    return code;
  };
  if (st != FR_OK) return give(st, f ? f->err : "setup failed");
  if (o.precision != FR_PREC_FP64 || full->in.viscous || full->in.PMG || full->in.motion)
    return give(FR_ERR_UNSUPPORTED, "parts: plain form (FP64), inviscid, static mesh, no P-multigrid");
  if (nparts > 1 && !nccl_api().ok) return give(FR_ERR_UNSUPPORTED, "libnccl.so.2 not found");
  std::vector<int> part;
  std::string e;
  if (nparts > full->E || !fr::partition_elements(full->mesh, nparts, part, e)) return give(FR_ERR_ARG, e);
  cudaStream_t stream = nullptr;
  if (cudaSetDevice(o.device) != cudaSuccess || cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) != cudaSuccess)
    return give(FR_ERR_CUDA, "stream create");
  p->ownStream = true;
  p->ownedStream = stream;
  if (!p->split_from(*full, part, rank, stream)) return give(FR_ERR_CUDA, p->err);
  p->opts.no_pdl = o.no_pdl;  // a part on its own stream may use PDL like any case
  p->usePdl = false;          // NCCL calls sit between its kernels
  p->comm = static_cast<ncclComm_t>(nccl_comm);
  for (size_t i = 0; i < p->cutPeer.size();) {
    size_t j = i;
    while (j < p->cutPeer.size() && p->cutPeer[j] == p->cutPeer[i]) j++;
    p->segPeer.push_back(p->cutPeer[i]);
    p->segOff.push_back((long long)i);
    p->segCount.push_back((long long)(j - i));
    i = j;
  }
  *out = p.release();
  return FR_OK;
}

int fr_part_nccl_ok(fr_case *c) {
  if (!c) return FR_ERR_ARG;
  return c->ncclOk ? FR_OK : FR_ERR_CUDA;
}

int fr_nccl_unique_id(void *id128) {
  if (!id128) return FR_ERR_ARG;
  if (!nccl_api().ok) return FR_ERR_UNSUPPORTED;
  ncclUniqueId u;
  if (nccl_api().uniqueId(&u) != ncclSuccess) return FR_ERR_CUDA;
  std::memcpy(id128, &u, sizeof(u));
  return FR_OK;
}

int fr_nccl_comm_init(int nranks, const void *id128, int rank, int device, void **comm) {
  if (!id128 || !comm || nranks < 1 || rank < 0 || rank >= nranks) return FR_ERR_ARG;
  if (!nccl_api().ok) return FR_ERR_UNSUPPORTED;
  if (cudaSetDevice(device) != cudaSuccess) return FR_ERR_CUDA;
  ncclUniqueId u;
  std::memcpy(&u, id128, sizeof(u));
  ncclComm_t c = nullptr;
  if (nccl_api().initRank(&c, nranks, u, rank) != ncclSuccess) return FR_ERR_CUDA;
  *comm = c;
  return FR_OK;
}

int fr_nccl_comm_destroy(void *comm) {
  if (!comm) return FR_ERR_ARG;
  if (!nccl_api().ok) return FR_ERR_UNSUPPORTED;
  return nccl_api().destroy(static_cast<ncclComm_t>(comm)) == ncclSuccess ? FR_OK : FR_ERR_CUDA;
}

const char *fr_shard_last_error(const fr_shard *s) { return s ? s->err.c_str() : "null shard"; }

void fr_shard_destroy(fr_shard *s) { delete s; }

int fr_shard_info(fr_shard *s, int *nparts, int *owned, long long *cut_points) {
  if (!s || !nparts) return FR_ERR_ARG;
  *nparts = (int)s->parts.size();
  for (size_t r = 0; r < s->parts.size(); r++) {
    if (owned) owned[r] = s->parts[r]->E;
    if (cut_points) cut_points[r] = s->parts[r]->cut.n;
  }
  return FR_OK;
}

namespace {
// whole-case array [nS][E][nF] <-> part r's [nS][E_r][nF]
void to_part(const fr_shard &s, int r, const double *U, std::vector<double> &out) {
  const fr_case &p = *s.parts[r];
  const int Ef = s.full->E, nS = p.nS, nF = p.nF;
  const auto &ow = s.owned[r];
  out.resize((size_t)nS * p.E * nF);
  for (int sp = 0; sp < nS; sp++)
    for (int el = 0; el < p.E; el++)
      std::memcpy(&out[((size_t)sp * p.E + el) * nF], &U[((size_t)sp * Ef + ow[el]) * nF], nF * sizeof(double));
}
void from_part(const fr_shard &s, int r, const std::vector<double> &in, double *U) {
  const fr_case &p = *s.parts[r];
  const int Ef = s.full->E, nS = p.nS, nF = p.nF;
  const auto &ow = s.owned[r];
  for (int sp = 0; sp < nS; sp++)
    for (int el = 0; el < p.E; el++)
      std::memcpy(&U[((size_t)sp * Ef + ow[el]) * nF], &in[((size_t)sp * p.E + el) * nF], nF * sizeof(double));
}
}  // namespace

int fr_shard_set_state(fr_shard *s, const double *U, size_t count) {
  if (!s || !U) return FR_ERR_ARG;
  const fr_case &F = *s->full;
  if (count != (size_t)F.nS * F.E * F.nF) return FR_ERR_ARG;
  frk::set_pdl(false);
  std::vector<double> buf;
  for (size_t r = 0; r < s->parts.size(); r++) {
    to_part(*s, (int)r, U, buf);
    if (!s->parts[r]->set_state_host(buf.data()) || !s->parts[r]->sync()) {
      s->err = s->parts[r]->err;
      return FR_ERR_CUDA;
    }
  }
  s->stateSet = true;
  return FR_OK;
}

int fr_shard_get_state(fr_shard *s, double *U, size_t count) {
  if (!s || !U) return FR_ERR_ARG;
  const fr_case &F = *s->full;
  if (count != (size_t)F.nS * F.E * F.nF) return FR_ERR_ARG;
  std::vector<double> buf;
  for (size_t r = 0; r < s->parts.size(); r++) {
    fr_case &p = *s->parts[r];
    buf.resize((size_t)p.nS * p.E * p.nF);
    if (!p.sync() || cudaMemcpy(buf.data(), p.U, buf.size() * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess) {
      s->err = "state read-back failed";
      return FR_ERR_CUDA;
    }
    from_part(*s, (int)r, buf, U);
  }
  return FR_OK;
}

int fr_shard_set_dt(fr_shard *s, double dt) {
  if (!s || !(dt > 0)) return FR_ERR_ARG;
  for (auto &p : s->parts)
    if (fr_set_dt(p.get(), dt) != FR_OK) {
      s->err = p->err;
      return FR_ERR_CUDA;
    }
  return FR_OK;
}

int fr_shard_calc_residual(fr_shard *s, int step) {
  if (!s) return FR_ERR_ARG;
  if (!s->stateSet) {
    s->err = "no state set";
    return FR_ERR_STATE;
  }
  if (step < 0 || step >= s->parts[0]->nRK) return FR_ERR_ARG;
  frk::set_pdl(false);
  return s->residual(step) && s->sync() ? FR_OK : FR_ERR_CUDA;
}

int fr_shard_get_residual(fr_shard *s, int step, double *divF, size_t count) {
  if (!s || !divF || step < 0 || step >= s->parts[0]->nRK) return FR_ERR_ARG;
  const fr_case &F = *s->full;
  if (count != (size_t)F.nS * F.E * F.nF) return FR_ERR_ARG;
  std::vector<double> buf;
  for (size_t r = 0; r < s->parts.size(); r++) {
    fr_case &p = *s->parts[r];
    buf.resize((size_t)p.nS * p.E * p.nF);
    if (!p.sync() ||
        cudaMemcpy(buf.data(), p.divF[step], buf.size() * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess) {
      s->err = "residual read-back failed";
      return FR_ERR_CUDA;
    }
    from_part(*s, (int)r, buf, divF);
  }
  return FR_OK;
}

int fr_shard_run(fr_shard *s, int nsteps) {
  if (!s || nsteps < 0) return FR_ERR_ARG;
  if (!s->stateSet) {
    s->err = "no state set";
    return FR_ERR_STATE;
  }
  frk::set_pdl(false);
  return s->run(nsteps) ? FR_OK : FR_ERR_CUDA;
}

int fr_shard_time(fr_shard *s, double *time, double *dt) {
  if (!s) return FR_ERR_ARG;
  fr_case &p = *s->parts[0];
  if (!s->sync()) return FR_ERR_CUDA;
  if (time) cudaMemcpy(time, p.timeAcc, sizeof(double), cudaMemcpyDeviceToHost);
  if (dt) cudaMemcpy(dt, p.dt, sizeof(double), cudaMemcpyDeviceToHost);
  return FR_OK;
}

int fr_synchronize(fr_case *c) {
  if (!c) return FR_ERR_ARG;
  if (c->hostOnly) {
    c->err = "host-only case: no device state";
    return FR_ERR_STATE;
  }
  return c->sync() ? FR_OK : FR_ERR_CUDA;
}

}  // extern "C"
