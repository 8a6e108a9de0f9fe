/*
 * Oracle harness around the reference solver (FlurryPP), compiled together with
 * the reference's own sources by oracle/Makefile into oracle/_ref/.
 *
 * TEST INFRASTRUCTURE ONLY.  It is the pinned CPU oracle (golden-vector
 * generator) and the timed CPU baseline.  The product library never links it.
 *
 * It drives the reference exactly as its driver does (src/flurry.cpp:127-174:
 * read deck -> setup -> initializeSolution -> loop { iter++; update(); [pmg
 * cycle] }), with three additions the benchmark cases need:
 *   - initial conditions the reference lacks (Mach-0.5 vortex, Taylor-Green
 *     vortex, seeded vortex) written straight into U_spts;
 *   - a seeded perturbation of interior mesh vertices before solver setup;
 *   - raw little-endian dumps of the state, operators, metrics, face
 *     connectivity and one residual evaluation's intermediates.
 *
 * usage: fr_ref_harness DECK OUTDIR [options]      (OUTDIR "-" = no dumps)
 *   --ic ref|vortex|tgv|uniform   initial condition (default ref = deck icType)
 *   --vortex EPS,XC,YC,MACH       vortex parameters (default 5,0,0,0.5)
 *   --tgv-mach M                  Taylor-Green Mach number (default 0.1)
 *   --perturb SEED,FRAC           perturb interior vertices by U(-FRAC h, FRAC h)
 *   --mu-inf MU                   override the non-dimensional viscosity
 *   --cfl-dt CFL                  fixed dt from the CFL formula on the IC
 *   --steps N                     time steps after the residual dump
 *   --time K,W                    W untimed then K timed steps, print JSON
 *   --time1 K                     after --time, K more steps timed on one
 *                                 OpenMP thread (the 1-thread figure)
 *   --threads T                   OpenMP threads (omp build)
 *   --monitors                    after the steps, calcResidual(0) and dump the
 *                                 wall-force coefficients writeResidual prints
 *                                 (wall_force [6]) and computeMassFlux for
 *                                 errorNorm 0, 1, 2 (mass_flux [3][nF])
 *   --error                       after the steps, dump solver::integrateError
 *                                 for errorNorm 0, 1, 2 (err_integrals [3][nF])
 *   --norms                       dump writeResidual's residual norms of the
 *                                 initial state's residual for resType 1, 2, 3
 *                                 (res_norms [3][nF]) and, after the steps, of
 *                                 the state's residual then (res_norms_final)
 *   --write-vtu PREFIX            after the steps, writeData with dataFileName
 *                                 PREFIX (the deck's plotType: 1 ParaView
 *                                 PREFIX_<iter>.vtu, 0 CSV PREFIX.csv.<iter>)
 */
#define private public
#define protected public
#include "solver.hpp"
#include "input.hpp"
#include "geo.hpp"
#include "multigrid.hpp"
#include "intFace.hpp"
#include "boundFace.hpp"
#include "ele.hpp"
#include "output.hpp"
#undef private
#undef protected

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <string>
#include <vector>
#ifdef _OMP
#include <omp.h>
#endif

extern "C" void fr_refshim_blas_threads(int n);

static std::string g_out;
static FILE *g_manifest = nullptr;

static void dump_raw(const char *name, const char *dtype, const void *p,
                     size_t elsize, const std::vector<size_t> &dims) {
  if (g_out == "-") return;
  size_t n = 1;
  for (size_t d : dims) n *= d;
  std::string path = g_out + "/" + name + ".bin";
  FILE *f = fopen(path.c_str(), "wb");
  if (!f) { fprintf(stderr, "cannot write %s\n", path.c_str()); exit(2); }
  if (n) fwrite(p, elsize, n, f);
  fclose(f);
  fprintf(g_manifest, "%s %s", name, dtype);
  for (size_t d : dims) fprintf(g_manifest, " %zu", d);
  fprintf(g_manifest, "\n");
  fflush(g_manifest);
}

static void dumpd(const char *name, const std::vector<double> &v,
                  const std::vector<size_t> &dims) {
  dump_raw(name, "f8", v.data(), sizeof(double), dims);
}
static void dumpi(const char *name, const std::vector<int> &v,
                  const std::vector<size_t> &dims) {
  dump_raw(name, "i4", v.data(), sizeof(int), dims);
}
template <typename A>
static void dumpA(const char *name, A &a, int rank) {
  std::vector<size_t> dims;
  for (int i = 0; i < rank; i++) dims.push_back(a.dims[i]);
  dumpd(name, a.data, dims);
}

struct Opts {
  std::string ic = "ref";
  double vEps = 5.0, vXc = 0.0, vYc = 0.0, vMach = 0.5;
  double tgvMach = 0.1;
  bool perturb = false;
  unsigned long long seed = 0;
  double frac = 0.0;
  bool muOverride = false;
  double mu = 0.0;
  double cflDt = -1.0;
  int steps = 0;
  int timeK = 0, timeW = 0, time1 = 0;
  int threads = 0;
  std::string vtu;
  bool error = false;
  bool monitors = false;
  bool norms = false;
};

/* Uniform double in [0,1) from the top 53 bits of a 64-bit Mersenne twister
 * draw.  The product library's mesh perturbation uses the same mapping. */
static double unit_draw(std::mt19937_64 &g) {
  return (double)(g() >> 11) * (1.0 / 9007199254740992.0);
}

static void perturb_vertices(geo &G, input &p, const Opts &o) {
  std::mt19937_64 g(o.seed);
  int nd = p.nDims;
  double h[3] = {(p.xmax - p.xmin) / p.nx, (p.ymax - p.ymin) / p.ny,
                 nd == 3 ? (p.zmax - p.zmin) / p.nz : 0.0};
  double lo[3] = {p.xmin, p.ymin, p.zmin}, hi[3] = {p.xmax, p.ymax, p.zmax};
  for (int v = 0; v < G.nVerts; v++) {
    bool interior = true;
    for (int d = 0; d < nd; d++) {
      double x = G.xv(v, d);
      double tol = 1e-9 * (hi[d] - lo[d]);
      if (std::fabs(x - lo[d]) < tol || std::fabs(x - hi[d]) < tol) interior = false;
    }
    if (!interior) continue;
    for (int d = 0; d < nd; d++) {
      double u = unit_draw(g);
      G.xv(v, d) += (2.0 * u - 1.0) * o.frac * h[d];
    }
  }
}

static void set_ic(solver &S, input &p, const Opts &o) {
  if (o.ic == "ref") return;
  const double gam = p.gamma;
  const int nd = p.nDims;
  const double PI = 3.141592653589793238462643383279502884;
  for (uint spt = 0; spt < S.nSpts; spt++) {
    for (uint e = 0; e < S.nEles; e++) {
      double x = S.pos_spts(spt, e, 0), y = S.pos_spts(spt, e, 1);
      double z = nd == 3 ? S.pos_spts(spt, e, 2) : 0.0;
      double rho, u, v, w = 0.0, pr;
      if (o.ic == "vortex") {
        double dx = x - o.vXc, dy = y - o.vYc;
        double f = 1.0 - (dx * dx + dy * dy);
        double eps = o.vEps;
        rho = std::pow(1.0 - eps * eps * (gam - 1.0) / (8.0 * gam * PI * PI) * std::exp(f),
                       1.0 / (gam - 1.0));
        u = o.vMach * std::sqrt(gam) - eps * dy / (2.0 * PI) * std::exp(0.5 * f);
        v = eps * dx / (2.0 * PI) * std::exp(0.5 * f);
        pr = std::pow(rho, gam);
      } else if (o.ic == "tgv") {
        double M = o.tgvMach;
        double p0 = 1.0 / (gam * M * M);
        u = std::sin(x) * std::cos(y) * std::cos(z);
        v = -std::cos(x) * std::sin(y) * std::cos(z);
        w = 0.0;
        pr = p0 + (std::cos(2.0 * x) + std::cos(2.0 * y)) * (std::cos(2.0 * z) + 2.0) / 16.0;
        rho = pr / p0;
      } else if (o.ic == "uniform") {
        rho = p.rhoBound; u = p.uBound; v = p.vBound; w = nd == 3 ? p.wBound : 0.0;
        pr = p.pBound;
      } else {
        fprintf(stderr, "unknown --ic %s\n", o.ic.c_str());
        exit(2);
      }
      S.U_spts(spt, e, 0) = rho;
      S.U_spts(spt, e, 1) = rho * u;
      S.U_spts(spt, e, 2) = rho * v;
      if (nd == 3) S.U_spts(spt, e, 3) = rho * w;
      S.U_spts(spt, e, nd + 1) = pr / (gam - 1.0) + 0.5 * rho * (u * u + v * v + w * w);
    }
  }
}

/* dt from the reference's element CFL formula (ele.cpp:1127-1146) evaluated
 * once on the current state, as solver::calcDt does (solver.cpp:447-468). */
static double cfl_dt(solver &S, input &p, double cfl) {
  double saveCFL = p.CFL;
  p.CFL = cfl;
  S.extrapolateU();
  for (auto &e : S.eles) e->calcWaveSpFpts();
  double dt = INFINITY;
  for (auto &e : S.eles) dt = std::min(dt, e->calcDt());
  p.CFL = saveCFL;
  return dt;
}

static void dump_setup(solver &S, input &p) {
  oper &op = S.opers[S.order];
  dumpA("opp_spts_to_fpts", op.opp_spts_to_fpts, 2);
  for (int d = 0; d < (int)S.nDims; d++) {
    char nm[64];
    snprintf(nm, sizeof nm, "opp_grad_spts_%d", d);
    dumpA(nm, op.opp_grad_spts[d], 2);
    snprintf(nm, sizeof nm, "opp_extrapolateFn_%d", d);
    dumpA(nm, op.opp_extrapolateFn[d], 2);
    if (p.viscous) {
      snprintf(nm, sizeof nm, "opp_correctU_%d", d);
      dumpA(nm, op.opp_correctU[d], 2);
    }
  }
  dumpA("opp_correction", op.opp_correction, 2);
  if (p.PMG) {
    dumpA("opp_prolong", op.opp_prolong, 2);
    if (S.order > 0) dumpA("opp_restrict", op.opp_restrict, 2);
  }
  dumpA("pos_spts", S.pos_spts, 3);
  dumpA("detJac_spts", S.detJac_spts, 2);
  dumpA("JGinv_spts", S.JGinv_spts, 4);
  dumpA("norm_fpts", S.norm_fpts, 3);
  dumpA("dA_fpts", S.dA_fpts, 2);
  dumpA("xv", S.Geo->xv, 2);

  /* Face table: one row per solver face (interior first, then boundary, as
   * geo::setupElesFaces builds them, geo.cpp:869-946). */
  int nF = (int)S.faces.size();
  int nPF = S.nDims == 2 ? S.order + 1 : (S.order + 1) * (S.order + 1);
  std::vector<int> ftype(nF), eL(nF), locL(nF), eR(nF), locR(nF), rot(nF), bc(nF);
  std::vector<int> fptR((size_t)nF * nPF, -1);
  for (int i = 0; i < nF; i++) {
    face *f = S.faces[i].get();
    ftype[i] = f->isBnd ? 1 : 0;
    eL[i] = f->eL->sID;
    locL[i] = f->locF_L;
    eR[i] = -1; locR[i] = -1; rot[i] = -1; bc[i] = -1;
    if (!f->isBnd) {
      intFace *g = dynamic_cast<intFace *>(f);
      eR[i] = g->eR->sID;
      locR[i] = g->faceID_R;
      rot[i] = g->relRot;
      for (int j = 0; j < nPF; j++) fptR[(size_t)i * nPF + j] = g->fptR[j];
    } else {
      boundFace *b = dynamic_cast<boundFace *>(f);
      bc[i] = b->bcType;
    }
  }
  dumpi("face_type", ftype, {(size_t)nF});
  dumpi("face_eL", eL, {(size_t)nF});
  dumpi("face_locL", locL, {(size_t)nF});
  dumpi("face_eR", eR, {(size_t)nF});
  dumpi("face_locR", locR, {(size_t)nF});
  dumpi("face_relRot", rot, {(size_t)nF});
  dumpi("face_bc", bc, {(size_t)nF});
  dumpi("face_fptR", fptR, {(size_t)nF, (size_t)nPF});
}

/* writeResidual's norm of divF_spts[0] (src/output.cpp:1011-1090): the
 * per-element ele::getNormResidual (src/ele.cpp:1922-1944) summed over the
 * elements (resType 1, 2) or their maximum (3), the square root for 2. */
static std::vector<double> residual_norms(solver &S, input &p) {
  std::vector<double> out;
  for (int rt = 1; rt <= 3; rt++) {
    std::vector<double> res(p.nFields, 0.0);
    for (auto &e : S.eles) {
      std::vector<double> r = e->getNormResidual(rt);
      for (int i = 0; i < p.nFields; i++) res[i] = rt == 3 ? std::max(res[i], r[i]) : res[i] + r[i];
    }
    if (rt == 2)
      for (auto &v : res) v = std::sqrt(v);
    out.insert(out.end(), res.begin(), res.end());
  }
  return out;
}

static void dump_residual_parts(solver &S, input &p) {
  dumpA("U_fpts", S.U_fpts, 3);
  dumpA("F_spts", S.F_spts, 4);
  dumpA("Fn_fpts", S.Fn_fpts, 3);
  dumpA("disFn_fpts", S.disFn_fpts, 3);
  dumpA("divF_0", S.divF_spts[0], 3);
  if (p.viscous) {
    dumpA("dU_spts", S.dU_spts, 4);
    dumpA("dU_fpts", S.dU_fpts, 4);
    dumpA("dUc_fpts", S.dUc_fpts, 3);
  }
  std::vector<double> ws;
  for (auto &e : S.eles)
    for (double w : e->waveSp_fpts) ws.push_back(w);
  dumpd("waveSp_fpts", ws, {S.nEles, S.nFpts});
}

int main(int argc, char **argv) {
  if (argc < 3) {
    fprintf(stderr, "usage: %s DECK OUTDIR [options]\n", argv[0]);
    return 2;
  }
  Opts o;
  for (int i = 3; i < argc; i++) {
    std::string a = argv[i];
    auto next = [&]() -> const char * {
      if (i + 1 >= argc) { fprintf(stderr, "missing value for %s\n", a.c_str()); exit(2); }
      return argv[++i];
    };
    if (a == "--ic") o.ic = next();
    else if (a == "--vortex") {
      if (sscanf(next(), "%lf,%lf,%lf,%lf", &o.vEps, &o.vXc, &o.vYc, &o.vMach) != 4) exit(2);
    } else if (a == "--tgv-mach") o.tgvMach = atof(next());
    else if (a == "--perturb") {
      o.perturb = true;
      if (sscanf(next(), "%llu,%lf", &o.seed, &o.frac) != 2) exit(2);
    } else if (a == "--mu-inf") { o.muOverride = true; o.mu = atof(next()); }
    else if (a == "--cfl-dt") o.cflDt = atof(next());
    else if (a == "--steps") o.steps = atoi(next());
    else if (a == "--time") {
      if (sscanf(next(), "%d,%d", &o.timeK, &o.timeW) != 2) exit(2);
    } else if (a == "--time1") o.time1 = atoi(next());
    else if (a == "--threads") o.threads = atoi(next());
    else if (a == "--write-vtu") o.vtu = next();
    else if (a == "--error") o.error = true;
    else if (a == "--monitors") o.monitors = true;
    else if (a == "--norms") o.norms = true;
    else { fprintf(stderr, "unknown option %s\n", a.c_str()); return 2; }
  }
  fr_refshim_blas_threads(1);
#ifdef _OMP
  if (o.threads > 0) omp_set_num_threads(o.threads);
#endif
  g_out = argv[2];
  if (g_out != "-") {
    std::string mf = g_out + "/manifest.txt";
    g_manifest = fopen(mf.c_str(), "w");
    if (!g_manifest) { fprintf(stderr, "cannot open %s\n", mf.c_str()); return 2; }
  }

  input params;
  params.readInputFile(argv[1]);
  if (o.muOverride) params.mu_inf = o.mu;

  solver S;
  multiGrid pmg;
  geo *G = nullptr;
  if (params.PMG) {
    if (o.perturb) { fprintf(stderr, "--perturb unsupported with PMG\n"); return 2; }
    pmg.setup(params.order, &params, S);
  } else {
    G = new geo;
    G->setup(&params);
    if (o.perturb) perturb_vertices(*G, params, o);
    S.setup(&params, params.order, G);
    S.initializeSolution();
  }
  set_ic(S, params, o);
  if (params.PMG && o.ic != "ref") {
    /* coarse levels start from their own IC; the cycle restricts the fine
     * state into them before first use (multigrid.cpp:169-173) */
  }
  if (params.dtType != 0 && o.ic != "ref") {
    /* initializeSolution computed the wave speeds on the deck's IC; redo it
     * on the state actually used (solver.cpp:1932-1938) */
    S.extrapolateU();
    for (auto &e : S.eles) e->calcWaveSpFpts();
  }
  if (o.cflDt > 0) {
    params.dt = cfl_dt(S, params, o.cflDt);
    params.dtType = 0;
    params.maxTime = 1e300;
  }

  if (g_manifest) {
    fprintf(g_manifest, "#meta nDims %u nFields %u order %d nEles %u nSpts %u nFpts %u nFaces %zu dt %.17g\n",
            S.nDims, S.nFields, S.order, S.nEles, S.nSpts, S.nFpts, S.faces.size(), params.dt);
    dumpA("U_init", S.U_spts, 3);
    dump_setup(S, params);
    /* one residual evaluation on the initial state (solver.cpp:366-445) */
    S.calcResidual(0);
    dump_residual_parts(S, params);
    if (o.norms) dumpd("res_norms", residual_norms(S, params), {3, (size_t)S.nFields});
  }

  if (o.steps > 0) {
    int &iter = params.iter;
    iter = params.initIter;
    for (int s = 0; s < o.steps; s++) {
      iter++;
      S.update();
      if (params.PMG) pmg.cycle(S);
    }
    dumpA("U_final", S.U_spts, 3);
    if (o.norms && g_manifest) {
      /* the residual of the final state, as the next writeResidual sees it */
      S.calcResidual(0);
      dumpd("res_norms_final", residual_norms(S, params), {3, (size_t)S.nFields});
    }
    std::vector<double> t = {params.time, params.dt};
    dumpd("time_dt", t, {2});
    if (params.dtType == 2) {
      std::vector<double> edt;
      for (auto &e : S.eles) edt.push_back(e->dt);
      dumpd("ele_dt", edt, {S.nEles});
    }
  }

  if (o.error && g_manifest) {
    std::vector<double> errs;
    for (int nrm = 0; nrm < 3; nrm++) {
      params.errorNorm = nrm;
      std::vector<double> e = S.integrateError();
      errs.insert(errs.end(), e.begin(), e.end());
    }
    dumpd("err_integrals", errs, {3, (size_t)S.nFields});
  }

  if (o.monitors && g_manifest) {
    S.calcResidual(0);
    /* src/output.cpp:1048-1066 */
    std::vector<double> force = S.computeWallForce();
    for (auto &f : force) f /= (0.5 * params.rhoBound * params.Uinf * params.Uinf);
    double alpha = std::atan2(params.vBound, params.uBound);
    std::vector<double> fTmp = force;
    force[0] = fTmp[0] * cos(alpha) + fTmp[1] * sin(alpha);
    force[1] = fTmp[1] * cos(alpha) - fTmp[0] * sin(alpha);
    if (params.viscous) {
      force[3] = fTmp[3] * cos(alpha) + fTmp[4] * sin(alpha);
      force[4] = fTmp[4] * cos(alpha) - fTmp[3] * sin(alpha);
    }
    dumpd("wall_force", force, {6});
    std::vector<double> flux;
    for (int nrm = 0; nrm < 3; nrm++) {
      params.errorNorm = nrm;
      std::vector<double> m = S.computeMassFlux();
      flux.insert(flux.end(), m.begin(), m.end());
    }
    dumpd("mass_flux", flux, {3, (size_t)S.nFields});
  }

  if (!o.vtu.empty()) {
    params.dataFileName = o.vtu;
    writeData(&S, &params);  /* plotType 1: ParaView, 0: CSV */
  }

  if (o.timeK > 0) {
    int &iter = params.iter;
    for (int s = 0; s < o.timeW; s++) { iter++; S.update(); if (params.PMG) pmg.cycle(S); }
    auto t0 = std::chrono::steady_clock::now();
    for (int s = 0; s < o.timeK; s++) { iter++; S.update(); if (params.PMG) pmg.cycle(S); }
    auto t1 = std::chrono::steady_clock::now();
    double sec = std::chrono::duration<double>(t1 - t0).count();
    double dof = (double)S.nSpts * S.nEles * S.nFields;
    double stages = (double)o.timeK * params.nRKSteps;
    int threads = 1;
#ifdef _OMP
    threads = omp_get_max_threads();
#endif
    double rate1 = 0.0, sec1 = 0.0;
    if (o.time1 > 0) {
#ifdef _OMP
      omp_set_num_threads(1);
#endif
      auto u0 = std::chrono::steady_clock::now();
      for (int s = 0; s < o.time1; s++) { iter++; S.update(); if (params.PMG) pmg.cycle(S); }
      auto u1 = std::chrono::steady_clock::now();
      sec1 = std::chrono::duration<double>(u1 - u0).count();
      rate1 = dof * (double)o.time1 * params.nRKSteps / sec1;
    }
    printf("{\"seconds\": %.6f, \"steps\": %d, \"stages\": %.0f, \"dof\": %.0f, "
           "\"dof_stage_per_s\": %.6e, \"threads\": %d, \"steps_1thread\": %d, "
           "\"seconds_1thread\": %.6f, \"dof_stage_per_s_1thread\": %.6e}\n",
           sec, o.timeK, stages, dof, dof * stages / sec, threads, o.time1, sec1, rate1);
  }
  if (g_manifest) fclose(g_manifest);
  return 0;
}
