// Solution files: the reference's ParaView (.vtu) and CSV writers and its
// restart reader, on host buffers that the device filled.
//
// The .vtu layout is the reference's own (src/output.cpp:137-512, the
// single-process branch): one <Piece> per element holding the (P+3)^d plot
// points — the element's corners, the flux points along its edges and faces,
// and its solution points, x fastest — with Density, Velocity and Pressure as
// ASCII with 16 significant digits, then the points and a structured split
// into (P+2)^d sub-cells.  The restart reader (src/solver.cpp:1789-1890,
// src/ele.cpp:1497-1921) takes the values at the solution points back out of
// that layout, converts them to conservative variables and, when the file's
// order differs from the case's, interpolates them to the case's points.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>

#include "fr_host.hpp"

namespace fr {

std::vector<Pt> loc_ppts(int nDims, int order, int ptsType) {
  // reference: src/points.cpp:164-196
  std::vector<double> p1 = pts1d(ptsType, order);
  p1.insert(p1.begin(), -1.0);
  p1.push_back(1.0);
  const int n = order + 3, nP = nDims == 2 ? n * n : n * n * n;
  std::vector<Pt> out(nP);
  for (int q = 0; q < nP; q++) {
    out[q].x = p1[q % n];
    out[q].y = p1[(q / n) % n];
    if (nDims == 3) out[q].z = p1[q / (n * n)];
  }
  return out;
}

std::vector<double> spts_to_ppts(int nDims, int order, int ptsType) {
  // reference: src/operators.cpp:145-165 (opp_spts_to_ppts)
  const std::vector<double> s1 = pts1d(ptsType, order);
  const auto pp = loc_ppts(nDims, order, ptsType);
  const int n = order + 1, nS = nDims == 2 ? n * n : n * n * n, nP = (int)pp.size();
  std::vector<double> A((size_t)nP * nS);
  for (int q = 0; q < nP; q++)
    for (int s = 0; s < nS; s++) {
      double v = lagrange(s1, pp[q].x, s % n) * lagrange(s1, pp[q].y, (s / n) % n);
      if (nDims == 3) v *= lagrange(s1, pp[q].z, s / (n * n));
      A[(size_t)q * nS + s] = v;
    }
  return A;
}

namespace {

// Appends "%.16g " for each value: the reference's ostream precision(16).
struct TextOut {
  std::FILE *f;
  std::vector<char> buf;
  size_t n = 0;
  explicit TextOut(std::FILE *fp) : f(fp), buf(1 << 20) {}
  void flush() {
    if (n) std::fwrite(buf.data(), 1, n, f);
    n = 0;
  }
  void room(size_t k) {
    if (n + k > buf.size()) flush();
  }
  void str(const char *s) {
    const size_t k = std::strlen(s);
    room(k);
    std::memcpy(buf.data() + n, s, k);
    n += k;
  }
  void num(double v) {
    room(32);
    n += (size_t)std::snprintf(buf.data() + n, 32, "%.16g ", v);
  }
  void fixed15(double v, char sep) {
    room(48);
    n += (size_t)std::snprintf(buf.data() + n, 48, "%.15f%c", v, sep);
  }
  void integer(long long v) {
    room(24);
    n += (size_t)std::snprintf(buf.data() + n, 24, "%lld ", v);
  }
};

}  // namespace

bool write_paraview(const std::string &path, int nDims, int order, int E, double time, long long iter,
                    const double *Vp, const double *pos, const double *gridVel, std::string &err) {
  std::FILE *f = std::fopen(path.c_str(), "wb");
  if (!f) {
    err = "cannot open " + path + " for writing";
    return false;
  }
  const int nF = nDims + 2, n1 = order + 3;
  const int nP = nDims == 2 ? n1 * n1 : n1 * n1 * n1;
  const int nSub = nDims == 2 ? (order + 2) * (order + 2) : (order + 2) * (order + 2) * (order + 2);
  TextOut o(f);
  char line[256];
  o.str("<?xml version=\"1.0\" ?>\n");
  o.str("<VTKFile type=\"UnstructuredGrid\" version=\"0.1\" byte_order=\"LittleEndian\" "
        "compressor=\"vtkZLibDataCompressor\">\n");
  std::snprintf(line, sizeof line, "<!-- TIME %.16g -->\n<!-- ITER %lld -->\n", time, iter);
  o.str(line);
  o.str("\t<UnstructuredGrid>\n");
  for (int e = 0; e < E; e++) {
    std::snprintf(line, sizeof line, "\t\t<Piece NumberOfPoints=\"%d\" NumberOfCells=\"%d\">\n", nP, nSub);
    o.str(line);
    o.str("\t\t\t<PointData>\n");
    auto V = [&](int q, int k) { return Vp[((size_t)q * E + e) * nF + k]; };
    o.str("\t\t\t\t<DataArray type=\"Float32\" Name=\"Density\" format=\"ascii\">\n");
    for (int q = 0; q < nP; q++) o.num(V(q, 0));
    o.str("\n\t\t\t\t</DataArray>\n");
    o.str("\t\t\t\t<DataArray type=\"Float32\" NumberOfComponents=\"3\" Name=\"Velocity\" format=\"ascii\">\n");
    for (int q = 0; q < nP; q++) {
      o.num(V(q, 1));
      o.num(V(q, 2));
      o.num(nDims == 2 ? 0.0 : V(q, 3));
    }
    o.str("\n\t\t\t\t</DataArray>\n");
    o.str("\t\t\t\t<DataArray type=\"Float32\" Name=\"Pressure\" format=\"ascii\">\n");
    for (int q = 0; q < nP; q++) o.num(V(q, nDims + 1));
    o.str("\n\t\t\t\t</DataArray>\n");
    if (gridVel) {  // moving mesh (src/output.cpp:383-399)
      o.str("\t\t\t\t<DataArray type=\"Float32\" NumberOfComponents=\"3\" Name=\"GridVelocity\" format=\"ascii\">\n");
      for (int q = 0; q < nP; q++) {
        for (int d = 0; d < nDims; d++) o.num(gridVel[((size_t)q * E + e) * nDims + d]);
        if (nDims == 2) o.num(0.0);
      }
      o.str("\n\t\t\t\t</DataArray>\n");
    }
    o.str("\t\t\t</PointData>\n");
    o.str("\t\t\t<Points>\n");
    o.str("\t\t\t\t<DataArray type=\"Float32\" NumberOfComponents=\"3\" format=\"ascii\">\n");
    for (int q = 0; q < nP; q++) {
      for (int d = 0; d < nDims; d++) o.num(pos[((size_t)q * E + e) * nDims + d]);
      if (nDims == 2) o.str("0 ");
    }
    o.str("\n\t\t\t\t</DataArray>\n");
    o.str("\t\t\t</Points>\n");
    o.str("\t\t\t<Cells>\n");
    o.str("\t\t\t\t<DataArray type=\"Int32\" Name=\"connectivity\" format=\"ascii\">\n");
    if (nDims == 2) {
      for (int j = 0; j < n1 - 1; j++)
        for (int i = 0; i < n1 - 1; i++) {
          o.integer(j * n1 + i);
          o.integer(j * n1 + i + 1);
          o.integer((j + 1) * n1 + i + 1);
          o.integer((j + 1) * n1 + i);
          o.str("\n");
        }
    } else {
      for (int k = 0; k < n1 - 1; k++)
        for (int j = 0; j < n1 - 1; j++)
          for (int i = 0; i < n1 - 1; i++) {
            for (int dk = 0; dk < 2; dk++) {
              o.integer(i + n1 * (j + n1 * (k + dk)));
              o.integer(i + 1 + n1 * (j + n1 * (k + dk)));
              o.integer(i + 1 + n1 * (j + 1 + n1 * (k + dk)));
              o.integer(i + n1 * (j + 1 + n1 * (k + dk)));
            }
            o.str("\n");
          }
    }
    o.str("\t\t\t\t</DataArray>\n");
    const int nv = nDims == 2 ? 4 : 8;
    o.str("\t\t\t\t<DataArray type=\"Int32\" Name=\"offsets\" format=\"ascii\">\n");
    for (int k = 0; k < nSub; k++) o.integer((long long)(k + 1) * nv);
    o.str("\n\t\t\t\t</DataArray>\n");
    o.str("\t\t\t\t<DataArray type=\"UInt8\" Name=\"types\" format=\"ascii\">\n");
    for (int k = 0; k < nSub; k++) o.integer(nDims == 2 ? 9 : 12);
    o.str("\n\t\t\t\t</DataArray>\n");
    o.str("\t\t\t</Cells>\n");
    o.str("\t\t</Piece>\n");
  }
  o.str("\t</UnstructuredGrid>\n");
  o.str("</VTKFile>\n");
  o.flush();
  const bool ok = std::ferror(f) == 0;
  if (std::fclose(f) != 0 || !ok) {
    err = "write error on " + path;
    return false;
  }
  return true;
}

bool write_csv(const std::string &path, int nDims, int nS, int nFp, int E, const double *U, const double *Ufpts,
               const double *posS, const double *posF, double gamma, std::string &err) {
  // reference: src/output.cpp:60-135 (header "rho,u,v,p" in 3-D too)
  std::FILE *f = std::fopen(path.c_str(), "wb");
  if (!f) {
    err = "cannot open " + path + " for writing";
    return false;
  }
  const int nF = nDims + 2;
  TextOut o(f);
  o.str("x,y,z,rho,u,v,p\n");
  auto row = [&](const double *x, const double *u) {
    for (int d = 0; d < nDims; d++) o.fixed15(x[d], ',');
    if (nDims == 2) o.str("0.0,");
    const double rho = u[0];
    double v2 = 0.0, v[3];
    for (int d = 0; d < nDims; d++) {
      v[d] = u[1 + d] / rho;
      v2 += v[d] * v[d];
    }
    o.fixed15(rho, ',');
    for (int d = 0; d < nDims; d++) o.fixed15(v[d], ',');
    o.fixed15((gamma - 1.0) * (u[nDims + 1] - 0.5 * rho * v2), '\n');
  };
  for (int e = 0; e < E; e++) {
    for (int s = 0; s < nS; s++) row(posS + ((size_t)s * E + e) * nDims, U + ((size_t)s * E + e) * nF);
    for (int q = 0; q < nFp; q++) row(posF + ((size_t)q * E + e) * nDims, Ufpts + ((size_t)q * E + e) * nF);
  }
  o.flush();
  const bool ok = std::ferror(f) == 0;
  if (std::fclose(f) != 0 || !ok) {
    err = "write error on " + path;
    return false;
  }
  return true;
}

namespace {

// The value between the first pair of double quotes in `s`, or "".
std::string quoted(const std::string &s) {
  const size_t a = s.find('"');
  if (a == std::string::npos) return "";
  const size_t b = s.find('"', a + 1);
  return b == std::string::npos ? "" : s.substr(a + 1, b - a - 1);
}

}  // namespace

bool read_restart_vtu(const std::string &path, const Input &in, int order, int E, std::vector<double> &U,
                      double &time, bool &hasTime, long long &iter, bool &hasIter, std::string &err) {
  std::ifstream f(path);
  if (!f.is_open()) {
    err = "Cannont open restart file.";  // the reference's message (src/solver.cpp:1810)
    return false;
  }
  const int nd = in.nDims, nF = in.nFields;
  const int n = order + 1, nS = nd == 2 ? n * n : n * n * n;
  U.assign((size_t)nS * E * nF, 0.0);
  hasTime = hasIter = false;
  std::string line, tok;
  bool grid = false;
  while (std::getline(f, line)) {
    std::istringstream ss(line);
    if (!(ss >> tok)) continue;
    if (tok == "<!--") {
      ss >> tok;
      if (tok == "TIME") hasTime = static_cast<bool>(ss >> time);
      else if (tok == "ITER") hasIter = static_cast<bool>(ss >> iter);
    } else if (tok == "<UnstructuredGrid>") {
      grid = true;
      break;
    }
  }
  if (!grid) {
    err = "Cannot find UnstructuredData tag in restart file.";
    return false;
  }
  int curR = -1;  // restart order whose interpolation matrix is in `interp`
  std::vector<double> interp, Ue;
  for (int e = 0; e < E; e++) {
    // <Piece NumberOfPoints="n" NumberOfCells="m">
    do {
      if (!std::getline(f, line)) {
        err = "restart file ends before element " + std::to_string(e);
        return false;
      }
    } while (line.find("<Piece") == std::string::npos);
    const size_t c = line.find("NumberOfCells");
    const int nCells = c == std::string::npos ? -1 : std::atoi(quoted(line.substr(c)).c_str());
    int r = -1;
    for (int k = 1; k <= 40 && r < 0; k++)
      if ((nd == 2 ? k * k : k * k * k) == nCells) r = k - 2;
    if (r < 0) {
      err = "restart element " + std::to_string(e) + ": cannot read its number of plot cells";
      return false;
    }
    const int nr = r + 1, nSr = nd == 2 ? nr * nr : nr * nr * nr, np = r + 3;
    const int nP = nd == 2 ? np * np : np * np * np;
    // plot-point index of each restart solution point
    std::vector<int> at(nSr);
    for (int s = 0; s < nSr; s++) {
      const int i = s % nr, j = (s / nr) % nr, k = s / (nr * nr);
      at[s] = nd == 2 ? (i + 1) + np * (j + 1) : (i + 1) + np * ((j + 1) + np * (k + 1));
    }
    std::vector<double> rho(nSr), vel((size_t)nSr * 3), p(nSr);
    bool fR = false, fV = false, fP = false;
    while (!(fR && fV && fP)) {
      if (!std::getline(f, line)) {
        err = "restart element " + std::to_string(e) + ": Density, Velocity and Pressure not all found";
        return false;
      }
      if (line.find("</Piece>") != std::string::npos) {
        err = "restart element " + std::to_string(e) + ": Density, Velocity and Pressure not all found";
        return false;
      }
      if (line.find("<DataArray") == std::string::npos) continue;
      const size_t nm = line.find("Name=");
      if (nm == std::string::npos) continue;
      const std::string name = quoted(line.substr(nm));
      const int comps = name == "Velocity" ? 3 : 1;
      if (name != "Density" && name != "Velocity" && name != "Pressure") continue;
      std::string data;
      if (!std::getline(f, data)) break;
      std::vector<double> vals;
      vals.reserve((size_t)nP * comps);
      const char *ptr = data.c_str();
      char *end = nullptr;
      for (;;) {
        const double v = std::strtod(ptr, &end);
        if (end == ptr) break;
        vals.push_back(v);
        ptr = end;
      }
      if ((int)vals.size() < nP * comps) {
        err = "restart element " + std::to_string(e) + ": short " + name + " array";
        return false;
      }
      for (int s = 0; s < nSr; s++) {
        const size_t q = (size_t)at[s] * comps;
        if (name == "Density") rho[s] = vals[q];
        else if (name == "Pressure") p[s] = vals[q];
        else
          for (int d = 0; d < 3; d++) vel[(size_t)s * 3 + d] = vals[q + d];
      }
      fR |= name == "Density";
      fV |= name == "Velocity";
      fP |= name == "Pressure";
    }
    while (line.find("</Piece>") == std::string::npos)
      if (!std::getline(f, line)) break;
    // conservative variables at the restart points (src/ele.cpp:1814-1825)
    Ue.assign((size_t)nSr * nF, 0.0);
    for (int s = 0; s < nSr; s++) {
      double *u = &Ue[(size_t)s * nF];
      u[0] = rho[s];
      double v2 = 0.0;
      for (int d = 0; d < nd; d++) {
        u[1 + d] = rho[s] * vel[(size_t)s * 3 + d];
        v2 += vel[(size_t)s * 3 + d] * vel[(size_t)s * 3 + d];
      }
      u[nd + 1] = p[s] / (in.gamma - 1) + 0.5 * rho[s] * v2;
    }
    if (r == order) {
      for (int s = 0; s < nS; s++)
        for (int k = 0; k < nF; k++) U[((size_t)s * E + e) * nF + k] = Ue[(size_t)s * nF + k];
      continue;
    }
    // another order: Lagrange interpolation in the restart file's point set
    // to the case's solution points (src/ele.cpp:1554-1596, 1902-1911)
    if (curR != r) {
      const std::vector<double> sr = pts1d(in.sptsTypeQuad, r), sf = pts1d(in.sptsTypeQuad, order);
      interp.assign((size_t)nS * nSr, 0.0);
      for (int s = 0; s < nS; s++)
        for (int q = 0; q < nSr; q++) {
          double v = lagrange(sr, sf[s % n], q % nr) * lagrange(sr, sf[(s / n) % n], (q / nr) % nr);
          if (nd == 3) v *= lagrange(sr, sf[s / (n * n)], q / (nr * nr));
          interp[(size_t)s * nSr + q] = v;
        }
      curR = r;
    }
    for (int s = 0; s < nS; s++)
      for (int k = 0; k < nF; k++) {
        double v = 0.0;
        for (int q = 0; q < nSr; q++) v += interp[(size_t)s * nSr + q] * Ue[(size_t)q * nF + k];
        U[((size_t)s * E + e) * nF + k] = v;
      }
  }
  return true;
}

}  // namespace fr
