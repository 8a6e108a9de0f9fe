// Deck reader and derived run-time values (reference: src/input.cpp).
#include <algorithm>
#include <cmath>
#include <fstream>
#include <map>
#include <sstream>

#include "fr_host.hpp"

namespace fr {

int bc_from_string(const std::string &s0) {
  std::string s = s0;
  std::transform(s.begin(), s.end(), s.begin(), ::tolower);
  static const std::map<std::string, int> m = {
      {"none", BC_NONE},
      {"fluid", BC_NONE},
      {"periodic", PERIODIC},
      {"char", CHAR_INOUT},
      {"sup_in", SUP_IN},
      {"sup_out", SUP_OUT},
      {"sub_in", SUB_IN},
      {"sub_out", SUB_OUT},
      {"slip_wall", SLIP_WALL},
      {"isothermal_noslip", ISOTHERMAL_NOSLIP},
      {"isothermal_noslip_moving", ISOTHERMAL_NOSLIP_MOVING},
      {"adiabatic_noslip", ADIABATIC_NOSLIP},
      {"symmetry", SYMMETRY}};
  auto it = m.find(s);
  return it == m.end() ? -100 : it->second;
}

namespace {

// Lines of the deck keyed by their first word; the first occurrence of a key
// wins, as in the reference's fileReader::getScalarValue (input.cpp:76-113).
struct Deck {
  std::map<std::string, std::string> first;
  std::vector<std::pair<std::string, std::string>> all;

  bool load(const std::string &path) {
    std::ifstream f(path);
    if (!f.is_open()) return false;
    std::string line;
    while (std::getline(f, line)) {
      std::stringstream ss(line);
      std::string key;
      if (!(ss >> key)) continue;
      std::string rest;
      std::getline(ss, rest);
      all.emplace_back(key, rest);
      if (!first.count(key)) first[key] = rest;
    }
    return true;
  }
  template <typename T>
  void get(const char *key, T &v) const {
    auto it = first.find(key);
    if (it == first.end()) return;
    std::stringstream ss(it->second);
    T tmp;
    if (ss >> tmp) v = tmp;
  }
  bool has(const char *key) const { return first.count(key) > 0; }
};

}  // namespace

bool read_deck(const std::string &path, Input &in, std::string &err) {
  Deck d;
  if (!d.load(path)) {
    err = "cannot open input file " + path;
    return false;
  }
  d.get("equation", in.equation);
  d.get("icType", in.icType);
  d.get("nDims", in.nDims);
  d.get("gamma", in.gamma);
  d.get("rhoBound", in.rhoBound);
  d.get("uBound", in.uBound);
  d.get("vBound", in.vBound);
  d.get("wBound", in.wBound);
  d.get("pBound", in.pBound);
  in.rhoIC = in.rhoBound;
  in.vxIC = in.uBound;
  in.vyIC = in.vBound;
  in.vzIC = in.wBound;
  in.pIC = in.pBound;
  if (in.icType == 0) {
    d.get("rhoIC", in.rhoIC);
    d.get("vxIC", in.vxIC);
    d.get("vyIC", in.vyIC);
    d.get("vzIC", in.vzIC);
    d.get("pIC", in.pIC);
  } else if (in.icType == 2) {
    d.get("vortexAngle", in.vortexAngle);
    d.get("vortexXmin", in.vortexXmin);
    d.get("vortexXmax", in.vortexXmax);
    d.get("vortexYmin", in.vortexYmin);
    d.get("vortexYmax", in.vortexYmax);
  }
  d.get("timeType", in.timeType);
  d.get("dtType", in.dtType);
  d.get("iterMax", in.iterMax);
  d.get("CFL", in.CFL);  // also kept for dtType 0, where fr_calc_dt may set dt once
  if (in.dtType != 0) {
    d.get("maxTime", in.maxTime);
    in.dt = 0;
  } else {
    d.get("dt", in.dt);
    in.maxTime = in.iterMax * in.dt;
  }
  d.get("viscous", in.viscous);
  d.get("motion", in.motion);
  if (in.motion == 4) {  // reference: src/input.cpp:324-332
    d.get("moveAx", in.moveAx);
    d.get("moveAy", in.moveAy);
    d.get("moveFx", in.moveFx);
    d.get("moveFy", in.moveFy);
  } else if (in.motion == 5) {
    d.get("moveAr", in.moveAr);
    d.get("moveFr", in.moveFr);
  }
  d.get("order", in.order);
  d.get("riemannType", in.riemannType);
  d.get("testCase", in.testCase);
  if (in.viscous) {
    // options the reference requires (no default) for viscous runs
    for (const char *k : {"Re", "MachBound", "MachWall"})
      if (!d.has(k)) {
        err = std::string("Required option not found: ") + k;
        return false;
      }
    in.penFact = 0.0;
    in.tau = 1.0;
    d.get("LDG_penFact", in.penFact);
    d.get("LDG_tau", in.tau);
    d.get("Re", in.Re);
    d.get("Lref", in.Lref);
    d.get("muGas", in.muGas);
    d.get("prandtl", in.prandtl);
    d.get("SGas", in.SGas);
    d.get("TGas", in.TGas);
    d.get("RGas", in.RGas);
    d.get("fixVis", in.fixVis);
    d.get("TBound", in.TBound);
    d.get("TWall", in.TWall);
    d.get("MachBound", in.MachBound);
    d.get("nxBound", in.nxBound);
    d.get("nyBound", in.nyBound);
    d.get("nzBound", in.nzBound);
    d.get("MachWall", in.MachWall);
    d.get("nxWall", in.nxWall);
    d.get("nyWall", in.nyWall);
    d.get("nzWall", in.nzWall);
  }
  d.get("restart", in.restart);
  if (in.restart) d.get("restartIter", in.restartIter);
  d.get("dataFileName", in.dataFileName);
  d.get("plotType", in.plotType);
  d.get("plotFreq", in.plotFreq);
  d.get("meshType", in.meshType);
  if (in.meshType == 1) {
    d.get("nx", in.nx);
    d.get("ny", in.ny);
    d.get("nz", in.nz);
    d.get("xmin", in.xmin);
    d.get("xmax", in.xmax);
    d.get("ymin", in.ymin);
    d.get("ymax", in.ymax);
    d.get("zmin", in.zmin);
    d.get("zmax", in.zmax);
    d.get("create_bcTop", in.create_bcTop);
    d.get("create_bcBottom", in.create_bcBottom);
    d.get("create_bcLeft", in.create_bcLeft);
    d.get("create_bcRight", in.create_bcRight);
    d.get("create_bcFront", in.create_bcFront);
    d.get("create_bcBack", in.create_bcBack);
  } else {
    d.get("meshFileName", in.meshFileName);
    for (auto &kv : d.all) {
      if (kv.first != "mesh_bound") continue;
      std::stringstream ss(kv.second);
      std::string a, b;
      if (ss >> a >> b) {
        std::transform(a.begin(), a.end(), a.begin(), ::tolower);
        std::transform(b.begin(), b.end(), b.begin(), ::tolower);
        in.meshBounds.emplace_back(a, b);
      }
    }
  }
  d.get("periodicDX", in.periodicDX);
  d.get("periodicDY", in.periodicDY);
  d.get("periodicDZ", in.periodicDZ);
  d.get("periodicTol", in.periodicTol);
  d.get("resType", in.resType);
  d.get("errorNorm", in.errorNorm);  // reference: src/input.cpp:424-425
  d.get("quadOrder", in.quadOrder);
  std::string spts = "Legendre";
  d.get("spts_type_quad", spts);
  if (spts == "Legendre")
    in.sptsTypeQuad = PTS_LEGENDRE;
  else if (spts == "Lobatto")
    in.sptsTypeQuad = PTS_LOBATTO;
  else {
    err = "unsupported spts_type_quad " + spts;
    return false;
  }
  d.get("vcjhSchemeQuad", in.vcjhSchemeQuad);
  d.get("PMG", in.PMG);
  if (in.PMG) {
    d.get("lowOrder", in.lowOrder);
    d.get("smoothSteps", in.smoothSteps);
  }
  return finalize_input(in, err);
}

bool finalize_input(Input &in, std::string &err) {
  if (in.equation != 1) {
    err = "only equation 1 (Euler/Navier-Stokes) is on the B200 path";
    return false;
  }
  if (in.nDims != 2 && in.nDims != 3) {
    err = "nDims must be 2 or 3";
    return false;
  }
  if (in.order < 0 || in.order > 5) {
    err = "order must be in 0..5";
    return false;
  }
  if (in.motion < 0 || in.motion > 5) {
    err = "motion must be 0 (static) or one of the reference's laws 1..5";
    return false;
  }
  if (in.motion != 0 && (in.viscous || in.riemannType != 0)) {
    err = "moving meshes run the inviscid Rusanov path";
    return false;
  }
  if (in.motion == 5 && in.nDims != 3) {
    err = "motion 5 (radial expansion) is 3-D only";  // reference: src/geo.cpp:208-216
    return false;
  }
  if (in.motion == 3 && in.nDims != 2) {
    err = "motion 3 is 2-D only";  // reference: src/geo.cpp:2775-2789
    return false;
  }
  if (in.riemannType == 1 && in.nDims == 3) {
    err = "Roe not implemented in 3D";  // reference: src/face.cpp:381
    return false;
  }
  in.nFields = in.nDims + 2;
  // RK tables (reference: src/input.cpp:469-505)
  switch (in.timeType) {
    case 0:
      in.nRKSteps = 1;
      in.RKa = {0.0};
      in.RKb = {1.0};
      break;
    case 2:
      in.nRKSteps = 2;
      in.RKa = {0.0, 1.0};
      in.RKb = {1.0 / 2.0, 1.0 / 2.0};
      break;
    case 4:
      in.nRKSteps = 4;
      in.RKa = {0.0, 0.5, 0.5, 1.0};
      in.RKb = {1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0};
      break;
    case 5:
      in.nRKSteps = 4;
      in.RKa = {0.0, 1.0 / 4.0, 1.0 / 3.0, 1.0 / 2.0, 1.0};
      in.RKb = {0.0};
      break;
    case 6:
      in.nRKSteps = 4;
      if (in.order <= 2)
        in.RKa = {0.0, 0.153, 0.442, 0.931, 1.0};
      else
        in.RKa = {0.0, 0.158, 0.477, 1.0, 1.0};
      in.RKb = {0.0};
      break;
    default:
      err = "Time-Stepping type not supported.";
      return false;
  }
  if (in.nDims == 2) in.wBound = 0;
  if (in.viscous && !in.nonDimensional) {
    in.nonDimensional = true;
    // Non-dimensionalisation (reference: src/input.cpp:521, 526-596)
    if (in.nDims == 2) in.nzBound = 0;
    double nMag = std::sqrt(in.nxBound * in.nxBound + in.nyBound * in.nyBound +
                            in.nzBound * in.nzBound);
    in.nxBound /= nMag;
    in.nyBound /= nMag;
    in.nzBound /= nMag;
    double Tref = in.TBound;
    double UBound = in.MachBound * std::sqrt(in.gamma * in.RGas * in.TBound);
    in.uBound = UBound * in.nxBound;
    in.vBound = UBound * in.nyBound;
    in.wBound = UBound * in.nzBound;
    in.muBound = in.muGas * std::pow(in.TBound / in.TGas, 1.5) *
                 ((in.TGas + in.SGas) / (in.TBound + in.SGas));
    in.rhoBound = in.muBound * in.Re / (UBound * in.Lref);
    in.pBound = in.rhoBound * in.RGas * in.TBound;
    double UWall = in.MachWall * std::sqrt(in.gamma * in.RGas * in.TWall);
    in.uWall = UWall * in.nxWall;
    in.vWall = UWall * in.nyWall;
    in.wWall = UWall * in.nzWall;
    double rhoRef = in.rhoBound;
    double pRef = rhoRef * UBound * UBound;
    double muRef = rhoRef * UBound * in.Lref;
    in.c_sth = in.SGas / in.TGas;
    in.mu_inf = in.muGas / muRef;
    in.rt_inf = in.TGas * in.RGas / (UBound * UBound);
    in.RGas = in.RGas * in.TBound / (UBound * UBound);
    in.rhoBound = 1.0;
    in.uBound = in.uBound / UBound;
    in.vBound = in.vBound / UBound;
    in.wBound = in.wBound / UBound;
    in.pBound = in.pBound / pRef;
    in.TWall = in.TWall / Tref;
    in.uWall /= UBound;
    in.vWall /= UBound;
    in.wWall /= UBound;
    in.rhoIC = in.rhoBound;
    in.vxIC = in.uBound;
    in.vyIC = in.vBound;
    in.vzIC = in.wBound;
    in.pIC = in.pBound;
  }
  return true;
}

}  // namespace fr
