// Cartesian mesh generation, face connectivity (hashing, O(n log n)),
// periodic pairing, flux-point orientation and metric terms.
#include <algorithm>
#include <cmath>
#include <fstream>
#include <map>
#include <random>
#include <set>
#include <sstream>
#include <unordered_map>

#include "fr_host.hpp"

namespace fr {

bool create_cartesian_mesh(const Input &in, Mesh &m, std::string &err) {
  // Vertex and element numbering follow src/geo.cpp:1477-1575.
  int nx = in.nx, ny = in.ny, nz = in.nDims == 2 ? 1 : in.nz;
  if (nx < 1 || ny < 1 || nz < 1) {
    err = "nx, ny, nz must be >= 1";
    return false;
  }
  m.nDims = in.nDims;
  double dx = (in.xmax - in.xmin) / nx, dy = (in.ymax - in.ymin) / ny,
         dz = (in.zmax - in.zmin) / nz;
  m.period[0] = in.xmax - in.xmin;
  m.period[1] = in.ymax - in.ymin;
  m.period[2] = in.nDims == 3 ? in.zmax - in.zmin : 1e300;
  m.periodicTol = in.periodicTol;
  int bcB = bc_from_string(in.create_bcBottom), bcR = bc_from_string(in.create_bcRight),
      bcT = bc_from_string(in.create_bcTop), bcL = bc_from_string(in.create_bcLeft),
      bcF = bc_from_string(in.create_bcFront), bcK = bc_from_string(in.create_bcBack);
  for (int b : {bcB, bcR, bcT, bcL, bcF, bcK})
    if (b == -100 || b == BC_NONE) {
      err = "unknown create_bc* boundary condition";
      return false;
    }
  m.bndFaceVerts.clear();
  m.bndFaceBc.clear();
  if (in.nDims == 2) {
    m.nVerts = (nx + 1) * (ny + 1);
    m.xv.resize((size_t)m.nVerts * 2);
    int nv = 0;
    for (int i = 0; i < ny + 1; i++)
      for (int j = 0; j < nx + 1; j++) {
        m.xv[2 * nv] = in.xmin + j * dx;
        m.xv[2 * nv + 1] = in.ymin + i * dy;
        nv++;
      }
    m.nEles = nx * ny;
    m.nNodes = 4;
    m.c2v.resize((size_t)m.nEles * 4);
    int e = 0;
    for (int i = 0; i < nx; i++)
      for (int j = 0; j < ny; j++) {
        int *c = &m.c2v[(size_t)4 * e++];
        c[0] = j * (nx + 1) + i;
        c[1] = j * (nx + 1) + i + 1;
        c[2] = (j + 1) * (nx + 1) + i + 1;
        c[3] = (j + 1) * (nx + 1) + i;
      }
    auto add = [&](int a, int b, int bc) {
      m.bndFaceVerts.push_back({a, b, -1, -1});
      m.bndFaceBc.push_back(bc);
    };
    for (int ix = 0; ix < nx; ix++) add(ix, ix + 1, bcB);
    for (int ix = 0; ix < nx; ix++) add((nx + 1) * ny + ix + 1, (nx + 1) * ny + ix, bcT);
    for (int iy = 0; iy < ny; iy++) add((iy + 1) * (nx + 1), iy * (nx + 1), bcL);
    for (int iy = 0; iy < ny; iy++) add(iy * (nx + 1) + nx, (iy + 1) * (nx + 1) + nx, bcR);
  } else {
    m.nVerts = (nx + 1) * (ny + 1) * (nz + 1);
    m.xv.resize((size_t)m.nVerts * 3);
    int nv = 0;
    for (int k = 0; k < nz + 1; k++)
      for (int j = 0; j < ny + 1; j++)
        for (int i = 0; i < nx + 1; i++) {
          m.xv[3 * nv] = in.xmin + i * dx;
          m.xv[3 * nv + 1] = in.ymin + j * dy;
          m.xv[3 * nv + 2] = in.zmin + k * dz;
          nv++;
        }
    m.nEles = nx * ny * nz;
    m.nNodes = 8;
    m.c2v.resize((size_t)m.nEles * 8);
    int e = 0;
    auto V = [&](int i, int j, int k) { return i + (nx + 1) * (j + (ny + 1) * k); };
    for (int k = 0; k < nz; k++)
      for (int i = 0; i < nx; i++)
        for (int j = 0; j < ny; j++) {
          int *c = &m.c2v[(size_t)8 * e++];
          c[0] = V(i, j, k);
          c[1] = V(i + 1, j, k);
          c[2] = V(i + 1, j + 1, k);
          c[3] = V(i, j + 1, k);
          c[4] = V(i, j, k + 1);
          c[5] = V(i + 1, j, k + 1);
          c[6] = V(i + 1, j + 1, k + 1);
          c[7] = V(i, j + 1, k + 1);
        }
    auto add = [&](int a, int b, int c, int d, int bc) {
      m.bndFaceVerts.push_back({a, b, c, d});
      m.bndFaceBc.push_back(bc);
    };
    for (int ix = 0; ix < nx; ix++)
      for (int iy = 0; iy < ny; iy++) {
        add(V(ix, iy, 0), V(ix + 1, iy, 0), V(ix + 1, iy + 1, 0), V(ix, iy + 1, 0), bcB);
        add(V(ix, iy, nz), V(ix + 1, iy, nz), V(ix + 1, iy + 1, nz), V(ix, iy + 1, nz), bcT);
      }
    for (int iz = 0; iz < nz; iz++)
      for (int iy = 0; iy < ny; iy++) {
        add(V(0, iy, iz), V(0, iy, iz + 1), V(0, iy + 1, iz + 1), V(0, iy + 1, iz), bcL);
        add(V(nx, iy, iz), V(nx, iy, iz + 1), V(nx, iy + 1, iz + 1), V(nx, iy + 1, iz), bcR);
      }
    for (int iz = 0; iz < nz; iz++)
      for (int ix = 0; ix < nx; ix++) {
        add(V(ix, 0, iz), V(ix, 0, iz + 1), V(ix + 1, 0, iz + 1), V(ix + 1, 0, iz), bcK);
        add(V(ix, ny, iz), V(ix, ny, iz + 1), V(ix + 1, ny, iz + 1), V(ix + 1, ny, iz), bcF);
      }
  }
  return true;
}

void perturb_interior_vertices(const Input &in, Mesh &m, uint64_t seed, double frac) {
  std::mt19937_64 g(seed);
  int nd = m.nDims;
  double h[3] = {(in.xmax - in.xmin) / in.nx, (in.ymax - in.ymin) / in.ny,
                 nd == 3 ? (in.zmax - in.zmin) / in.nz : 0.0};
  double lo[3] = {in.xmin, in.ymin, in.zmin}, hi[3] = {in.xmax, in.ymax, in.zmax};
  for (int v = 0; v < m.nVerts; v++) {
    bool interior = true;
    for (int d = 0; d < nd; d++) {
      double x = m.xv[(size_t)v * nd + d];
      double tol = 1e-9 * (hi[d] - lo[d]);
      if (std::fabs(x - lo[d]) < tol || std::fabs(x - hi[d]) < tol) interior = false;
    }
    if (!interior) continue;
    for (int d = 0; d < nd; d++) {
      double u = (double)(g() >> 11) * (1.0 / 9007199254740992.0);
      m.xv[(size_t)v * nd + d] += (2.0 * u - 1.0) * frac * h[d];
    }
  }
}

namespace {

// Nodes of a Gmsh volume cell on the path: Lagrange quads (4, 9, 16, ...,
// 121 nodes), Lagrange hexes (8, 27, 64, 125, 216) and the 20-node
// serendipity hex (reference: src/geo.cpp:1160-1353).  -2: a simplex or prism
// that the reference reads as a collapsed quad or hex; -1: unknown.
int gmsh_cell_nodes(int type, int nd) {
  if (nd == 2) {
    switch (type) {
      case 3: return 4;
      case 10: return 9;
      case 16: return 8;  // serendipity quad: refused by the shape functions
      case 36: return 16;
      case 37: return 25;
      case 38: return 36;
      case 47: return 49;
      case 48: return 64;
      case 49: return 81;
      case 50: return 100;
      case 51: return 121;
      case 2: case 9: return -2;
    }
  } else {
    switch (type) {
      case 5: return 8;
      case 17: return 20;
      case 12: return 27;
      case 92: return 64;
      case 93: return 125;
      case 94: return 216;
      case 4: case 6: return -2;
    }
  }
  return -1;
}

// Nodes of a boundary element that join its boundary's point set: every node
// of an edge, the corners of a quad face (reference: src/geo.cpp:1388-1436).
int gmsh_face_points(int type) {
  switch (type) {
    case 1: return 2;
    case 2: return 3;
    case 3: case 10: case 16: case 36: case 37: case 38: return 4;
    case 8: return 3;
    case 26: return 4;
    case 27: return 5;
    case 28: return 6;
    case 62: return 7;
    case 63: return 8;
    case 64: return 9;
    case 65: return 10;
    case 66: return 11;
  }
  return -1;
}

}  // namespace

bool read_gmsh(const std::string &path, Input &in, Mesh &m, std::string &err) {
  std::ifstream f(path);
  if (!f.is_open()) {
    err = "Unable to open mesh file " + path;
    return false;
  }
  std::string line;
  auto seek = [&](const char *tag) {
    f.clear();
    f.seekg(0, std::ios::beg);
    while (std::getline(f, line))
      if (line.find(tag) != std::string::npos) return true;
    return false;
  };
  // $PhysicalNames: boundary tag -> boundary index (in file order) and BC
  if (!seek("$PhysicalNames")) {
    err = "$PhysicalNames tag not found in Gmsh file!";
    return false;
  }
  int nNames = 0;
  f >> nNames;
  std::getline(f, line);
  std::map<int, int> tag2bnd;  // -1: fluid
  std::vector<int> bndBc;
  int nd = in.nDims;
  for (int i = 0; i < nNames; i++) {
    std::getline(f, line);
    std::stringstream ss(line);
    int dim, id;
    std::string name;
    ss >> dim >> id >> name;
    name.erase(std::remove(name.begin(), name.end(), '"'), name.end());
    std::transform(name.begin(), name.end(), name.begin(), ::tolower);
    std::string bcName;
    for (auto &kv : in.meshBounds)
      if (kv.first == name) bcName = kv.second;
    if (bcName.empty()) {
      err = "Unrecognized mesh boundary: \"" + name + "\"";
      return false;
    }
    if (bcName == "fluid") {
      nd = dim;
      tag2bnd[id] = -1;
      continue;
    }
    int bc = bc_from_string(bcName);
    if (bc == -100 || bc == BC_NONE) {
      err = "Unrecognized boundary condition: \"" + bcName + "\"";
      return false;
    }
    tag2bnd[id] = (int)bndBc.size();
    bndBc.push_back(bc);
  }
  in.nDims = nd;
  m.nDims = nd;
  // $Nodes: positions in file order (node ids are assumed 1..n in order)
  if (!seek("$Nodes")) {
    err = "$Nodes tag not found in Gmsh file!";
    return false;
  }
  f >> m.nVerts;
  std::getline(f, line);
  m.xv.assign((size_t)m.nVerts * nd, 0.0);
  for (int i = 0; i < m.nVerts; i++) {
    std::getline(f, line);
    std::stringstream ss(line);
    long long id;
    ss >> id;
    for (int d = 0; d < nd; d++) ss >> m.xv[(size_t)i * nd + d];
  }
  if (!seek("$Elements")) {
    err = "$Elements tag not found in Gmsh file!";
    return false;
  }
  long long nEl = 0;
  f >> nEl;
  std::getline(f, line);
  std::vector<std::set<int>> pts(bndBc.size());
  m.nNodes = 0;
  m.c2v.clear();
  m.nEles = 0;
  for (long long k = 0; k < nEl; k++) {
    std::getline(f, line);
    std::stringstream ss(line);
    int id, type, nTags, tag0 = 0, tmp;
    ss >> id >> type >> nTags;
    if (nTags > 0) ss >> tag0;
    for (int t = 1; t < nTags; t++) ss >> tmp;
    auto it = tag2bnd.find(tag0);
    if (it == tag2bnd.end()) {
      err = "element with an unknown physical tag";
      return false;
    }
    if (it->second == -1) {
      const int nv = gmsh_cell_nodes(type, nd);
      if (nv == -2) {
        err = "Gmsh element type " + std::to_string(type) +
              " (triangle, tetrahedron or prism read as a collapsed quad or hex) is not on the B200 path";
        return false;
      }
      if (nv < 0) {
        err = "Gmsh element ID " + std::to_string(k) + ", type " + std::to_string(type) +
              ": element type not recognized";
        return false;
      }
      if (m.nNodes == 0) m.nNodes = nv;
      if (nv != m.nNodes) {
        err = "elements with different node counts in one mesh (" + std::to_string(m.nNodes) + " and " +
              std::to_string(nv) + ")";
        return false;
      }
      int g[216];
      for (int v = 0; v < nv; v++) ss >> g[v];
      if (type == 17) {
        // Gmsh lists the 20-node hex's mid-edge nodes by edge 0-1, 0-3, 0-4,
        // 1-2, 1-5, 2-3, 2-6, 3-7, 4-5, 4-7, 5-6, 6-7; the serendipity shape
        // functions number them 0-1, 1-2, 2-3, 3-0, 0-4, 1-5, 2-6, 3-7, 4-5,
        // 5-6, 6-7, 7-4 (reference: src/geo.cpp:1284-1294)
        static const int slot[12] = {8, 11, 12, 9, 13, 10, 14, 15, 16, 19, 17, 18};
        int h[20];
        for (int v = 0; v < 8; v++) h[v] = g[v];
        for (int v = 0; v < 12; v++) h[slot[v]] = g[8 + v];
        for (int v = 0; v < 20; v++) g[v] = h[v];
      }
      for (int v = 0; v < nv; v++) m.c2v.push_back(g[v] - 1);
      m.nEles++;
    } else {
      const int np = gmsh_face_points(type);
      if (np < 0) {
        err = "Boundary Element (Face) Type Not Recognized!";
        return false;
      }
      for (int v = 0; v < np; v++) {
        int g;
        ss >> g;
        pts[it->second].insert(g - 1);
      }
    }
  }
  if (m.nEles == 0) {
    err = "no fluid elements in the Gmsh file";
    return false;
  }
  m.bndFaceVerts.clear();
  m.bndFaceBc.clear();
  m.bndPointSets.clear();
  m.bndPointBc = bndBc;
  for (auto &p : pts) m.bndPointSets.emplace_back(p.begin(), p.end());
  m.period[0] = in.periodicDX;
  m.period[1] = in.periodicDY;
  m.period[2] = in.periodicDZ;
  m.periodicTol = in.periodicTol;
  return true;
}

namespace {

// Local face -> element vertices, in the order that the element's flux
// points run over the face (reference: src/geo.cpp:375-381 for the vertex sets).
const int kQuadFace[4][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}};
const int kHexFace[6][4] = {{0, 1, 2, 3}, {4, 5, 6, 7}, {3, 0, 4, 7},
                            {2, 1, 5, 6}, {1, 0, 4, 5}, {3, 2, 6, 7}};

struct Key4 {
  int v[4];
  bool operator==(const Key4 &o) const {
    return v[0] == o.v[0] && v[1] == o.v[1] && v[2] == o.v[2] && v[3] == o.v[3];
  }
};
struct Key4Hash {
  size_t operator()(const Key4 &k) const {
    uint64_t h = 1469598103934665603ull;
    for (int i = 0; i < 4; i++) {
      h ^= (uint64_t)(uint32_t)k.v[i];
      h *= 1099511628211ull;
    }
    return (size_t)h;
  }
};

Key4 face_key(const Mesh &m, int e, int f) {
  Key4 k{{-1, -1, -1, -1}};
  int nfv = m.nDims == 2 ? 2 : 4;
  for (int i = 0; i < nfv; i++) {
    int lv = m.nDims == 2 ? kQuadFace[f][i] : kHexFace[f][i];
    k.v[i] = m.c2v[(size_t)e * m.nNodes + lv];
  }
  std::sort(k.v, k.v + nfv);
  return k;
}

// Geometric shape functions (reference: src/funcs.cpp:145-1015).  Lagrange
// quads of (n+1)^2 nodes and hexes of (n+1)^3 nodes interpolate on n+1
// equidistant points per direction; their nodes are numbered shell by shell
// from the outside in: corners, then the points inside each edge, then (hexes)
// the points inside each face, each face numbered like a quad, then the next
// shell; an odd count ends with the centre.  This is Gmsh's numbering, which
// the reference reads unchanged.  The 20-node serendipity hex has corners
// 0-7, then the mid-edge nodes of the bottom ring (8-11: edges 0-1, 1-2, 2-3,
// 3-0), the vertical edges (12-15: above nodes 0-3) and the top ring (16-19).
const double kHexXi[8] = {-1, 1, 1, -1, -1, 1, 1, -1};
const double kHexEta[8] = {-1, -1, 1, 1, -1, -1, 1, 1};
const double kHexMu[8] = {-1, -1, -1, -1, 1, 1, 1, 1};

struct ShapeFn {
  int nd = 2, nNodes = 4;
  bool serendipity = false;
  std::vector<double> xl;              // equidistant 1-D nodes on [-1, 1]
  std::vector<std::array<int, 3>> ijk;  // per node: 1-D index along xi, eta, mu

  // (a, b) pairs of a quad's nodes whose 1-D indices run over [lo, hi]
  static void quad_rings(int lo, int hi, std::vector<std::array<int, 2>> &out) {
    const int n = hi - lo + 1;
    for (int l = 0; l < n / 2; l++) {
      const int a = lo + l, b = hi - l, m = n - 2 * (l + 1);
      out.push_back({a, a});
      out.push_back({b, a});
      out.push_back({b, b});
      out.push_back({a, b});
      for (int k = 0; k < m; k++) out.push_back({a + 1 + k, a});
      for (int k = 0; k < m; k++) out.push_back({b, a + 1 + k});
      for (int k = 0; k < m; k++) out.push_back({b - 1 - k, b});
      for (int k = 0; k < m; k++) out.push_back({a, b - 1 - k});
    }
    if (n % 2) out.push_back({lo + n / 2, lo + n / 2});
  }

  bool init(int nDims, int nodes, std::string &err) {
    nd = nDims;
    nNodes = nodes;
    serendipity = nd == 3 && nodes == 20;
    ijk.clear();
    if (serendipity) return true;
    int nSide = 1;
    while (nSide * nSide * (nd == 3 ? nSide : 1) < nodes) nSide++;
    if (nSide < 2 || nSide * nSide * (nd == 3 ? nSide : 1) != nodes) {
      err = nd == 2 ? "For Lagrange quad of order N, must have (N+1)^2 shape points."
                    : "For Lagrange hex of order N, must have (N+1)^3 shape points.";
      return false;
    }
    xl.resize(nSide);
    const double dxi = 2. / (nSide - 1);
    for (int i = 0; i < nSide; i++) xl[i] = -1. + i * dxi;
    if (nd == 2) {
      std::vector<std::array<int, 2>> q;
      quad_rings(0, nSide - 1, q);
      for (auto &ab : q) ijk.push_back({ab[0], ab[1], 0});
      return true;
    }
    for (int l = 0; l < nSide / 2; l++) {
      const int i = l, i2 = nSide - 1 - l, m = nSide - 2 * (l + 1);
      const int c[8][3] = {{i, i, i},   {i2, i, i},   {i2, i2, i},   {i, i2, i},
                           {i, i, i2},  {i2, i, i2},  {i2, i2, i2},  {i, i2, i2}};
      for (auto &v : c) ijk.push_back({v[0], v[1], v[2]});
      // edges 0-1, 0-3, 0-4, 1-2, 1-5, 2-3, 2-6, 3-7, 4-5, 4-7, 5-6, 6-7
      for (int e = 0; e < 12; e++)
        for (int k = 0; k < m; k++) {
          const int r = i + 1 + k, rr = i2 - 1 - k;
          const int t[12][3] = {{r, i, i},  {i, r, i},   {i, i, r},  {i2, r, i},  {i2, i, r},  {rr, i2, i},
                                {i2, i2, r}, {i, i2, r}, {r, i, i2}, {i, r, i2}, {i2, r, i2}, {rr, i2, i2}};
          ijk.push_back({t[e][0], t[e][1], t[e][2]});
        }
      // faces mu=lo, eta=lo, xi=lo, xi=hi, eta=hi, mu=hi, each a quad's rings
      std::vector<std::array<int, 2>> q;
      quad_rings(i + 1, i2 - 1, q);
      for (auto &ab : q) ijk.push_back({ab[1], ab[0], i});
      for (auto &ab : q) ijk.push_back({ab[0], i, ab[1]});
      for (auto &ab : q) ijk.push_back({i, ab[1], ab[0]});
      for (auto &ab : q) ijk.push_back({i2, ab[0], ab[1]});
      for (auto &ab : q) ijk.push_back({nSide - 1 - ab[0], i2, ab[1]});
      for (auto &ab : q) ijk.push_back({ab[0], ab[1], i2});
    }
    if (nSide % 2) ijk.push_back({nSide / 2, nSide / 2, nSide / 2});
    return (int)ijk.size() == nodes;
  }

  // mid-edge node n of the serendipity hex: the varying direction and the
  // sides of the other two (in xi, eta, mu order with the varying one skipped)
  static void ser_edge(int n, int &axis, double &s1, double &s2) {
    static const int ax[12] = {0, 1, 0, 1, 2, 2, 2, 2, 0, 1, 0, 1};
    static const double a1[12] = {-1, 1, 1, -1, -1, 1, 1, -1, -1, 1, 1, -1};
    static const double a2[12] = {-1, -1, -1, -1, -1, -1, 1, 1, 1, 1, 1, 1};
    axis = ax[n - 8];
    s1 = a1[n - 8];
    s2 = a2[n - 8];
  }

  void eval(const Pt &p, double *N) const {
    const double x[3] = {p.x, p.y, p.z};
    if (serendipity) {
      for (int n = 0; n < 8; n++) {
        const double sx = kHexXi[n], sy = kHexEta[n], sz = kHexMu[n];
        N[n] = .125 * (1 + x[0] * sx) * (1 + x[1] * sy) * (1 + x[2] * sz) * (x[0] * sx + x[1] * sy + x[2] * sz - 2);
      }
      for (int n = 8; n < 20; n++) {
        int a;
        double s1, s2;
        ser_edge(n, a, s1, s2);
        const int b = a == 0 ? 1 : 0, c = a == 2 ? 1 : 2;
        N[n] = .25 * (1 - x[a] * x[a]) * (1 + x[b] * s1) * (1 + x[c] * s2);
      }
      return;
    }
    for (int n = 0; n < nNodes; n++) {
      double v = lagrange(xl, x[0], ijk[n][0]) * lagrange(xl, x[1], ijk[n][1]);
      if (nd == 3) v *= lagrange(xl, x[2], ijk[n][2]);
      N[n] = v;
    }
  }

  void deval(const Pt &p, double *dN /*[nNodes][nd]*/) const {
    const double x[3] = {p.x, p.y, p.z};
    if (serendipity) {
      for (int n = 0; n < 8; n++) {
        const double s[3] = {kHexXi[n], kHexEta[n], kHexMu[n]};
        for (int d = 0; d < 3; d++) {
          const int b = d == 0 ? 1 : 0, c = d == 2 ? 1 : 2;
          dN[3 * n + d] = .125 * s[d] * (1 + x[b] * s[b]) * (1 + x[c] * s[c]) *
                          (2 * x[d] * s[d] + x[b] * s[b] + x[c] * s[c] - 1);
        }
      }
      for (int n = 8; n < 20; n++) {
        int a;
        double s1, s2;
        ser_edge(n, a, s1, s2);
        const int b = a == 0 ? 1 : 0, c = a == 2 ? 1 : 2;
        dN[3 * n + a] = -.5 * x[a] * (1 + x[b] * s1) * (1 + x[c] * s2);
        dN[3 * n + b] = .25 * (1 - x[a] * x[a]) * s1 * (1 + x[c] * s2);
        dN[3 * n + c] = .25 * (1 - x[a] * x[a]) * (1 + x[b] * s1) * s2;
      }
      return;
    }
    for (int n = 0; n < nNodes; n++) {
      const double L0 = lagrange(xl, x[0], ijk[n][0]), L1 = lagrange(xl, x[1], ijk[n][1]);
      const double D0 = dlagrange(xl, x[0], ijk[n][0]), D1 = dlagrange(xl, x[1], ijk[n][1]);
      if (nd == 2) {
        dN[2 * n + 0] = D0 * L1;
        dN[2 * n + 1] = L0 * D1;
      } else {
        const double L2 = lagrange(xl, x[2], ijk[n][2]), D2 = dlagrange(xl, x[2], ijk[n][2]);
        dN[3 * n + 0] = D0 * L1 * L2;
        dN[3 * n + 1] = L0 * D1 * L2;
        dN[3 * n + 2] = L0 * L1 * D2;
      }
    }
  }
};
}  // namespace

bool shape_supported(int nDims, int nNodes) {
  ShapeFn sf;
  std::string err;
  return (nDims == 2 || nDims == 3) && nNodes >= 4 && nNodes <= 216 && sf.init(nDims, nNodes, err);
}

bool shape_tables(int nDims, int nNodes, const std::vector<Pt> &loc, std::vector<double> &N,
                  std::vector<double> &dN, std::string &err) {
  ShapeFn sf;
  if (!sf.init(nDims, nNodes, err)) return false;
  N.assign(loc.size() * nNodes, 0.0);
  dN.assign(loc.size() * nNodes * nDims, 0.0);
  for (size_t q = 0; q < loc.size(); q++) {
    sf.eval(loc[q], &N[q * nNodes]);
    sf.deval(loc[q], &dN[q * nNodes * nDims]);
  }
  return true;
}

bool positions_at(const Mesh &m, const std::vector<Pt> &loc, std::vector<double> &pos, std::string &err) {
  ShapeFn sf;
  if (!sf.init(m.nDims, m.nNodes, err)) return false;
  const int nd = m.nDims, nN = m.nNodes, E = m.nEles, nP = (int)loc.size();
  std::vector<double> N((size_t)nP * nN);
  for (int q = 0; q < nP; q++) sf.eval(loc[q], &N[(size_t)q * nN]);
  pos.assign((size_t)nP * E * nd, 0.0);
  for (int e = 0; e < E; e++) {
    const int *cv = &m.c2v[(size_t)e * nN];
    for (int q = 0; q < nP; q++)
      for (int d = 0; d < nd; d++) {
        double x = 0.0;
        for (int k = 0; k < nN; k++) x += N[(size_t)q * nN + k] * m.xv[(size_t)cv[k] * nd + d];
        pos[((size_t)q * E + e) * nd + d] = x;
      }
  }
  return true;
}

bool build_faces(const Mesh &m, int order, int ptsType, std::vector<Face> &faces, std::string &err) {
  const int nd = m.nDims;
  const int nLocF = nd == 2 ? 4 : 6;
  const int n1 = order + 1;
  const int nPF = nd == 2 ? n1 : n1 * n1;
  faces.clear();
  if ((int)m.xv.size() < m.nVerts * nd || m.c2v.size() != (size_t)m.nEles * m.nNodes) {
    err = "mesh arrays do not match their sizes";
    return false;
  }
  for (int v : m.c2v)
    if (v < 0 || v >= m.nVerts) {
      err = "element node index out of range";
      return false;
    }
  ShapeFn sf;
  if (!sf.init(nd, m.nNodes, err)) return false;
  const int nN = m.nNodes;

  // Boundary-face BC lookup by sorted vertex list.
  std::unordered_map<Key4, int, Key4Hash> bndBc;
  for (size_t i = 0; i < m.bndFaceVerts.size(); i++) {
    Key4 k{{m.bndFaceVerts[i][0], m.bndFaceVerts[i][1], m.bndFaceVerts[i][2], m.bndFaceVerts[i][3]}};
    std::sort(k.v, k.v + (nd == 2 ? 2 : 4));
    bndBc[k] = m.bndFaceBc[i];
  }

  // Pair element faces through their sorted vertex lists.
  struct Side {
    int e, f;
  };
  std::unordered_map<Key4, std::pair<Side, Side>, Key4Hash> seen;
  seen.reserve((size_t)m.nEles * nLocF);
  for (int e = 0; e < m.nEles; e++)
    for (int f = 0; f < nLocF; f++) {
      Key4 k = face_key(m, e, f);
      auto it = seen.find(k);
      if (it == seen.end()) {
        seen.emplace(k, std::make_pair(Side{e, f}, Side{-1, -1}));
      } else {
        if (it->second.second.e != -1) {
          err = "more than 2 cells share a face";
          return false;
        }
        it->second.second = Side{e, f};
      }
    }

  // Interior faces in (element, local face) order of their first side.
  std::vector<std::pair<Side, Side>> interior;
  std::vector<std::pair<Side, int>> boundary;  // side, bc
  for (int e = 0; e < m.nEles; e++)
    for (int f = 0; f < nLocF; f++) {
      Key4 k = face_key(m, e, f);
      auto &pr = seen[k];
      if (pr.first.e != e || pr.first.f != f) continue;  // emitted once, at first side
      if (pr.second.e >= 0) {
        interior.push_back(pr);
      } else if (!m.bndPointSets.empty()) {
        // first boundary holding every vertex of the face
        int nfv = nd == 2 ? 2 : 4, bc = -100;
        for (size_t bi = 0; bi < m.bndPointSets.size() && bc == -100; bi++) {
          bool all = true;
          for (int q = 0; q < nfv && all; q++)
            all = std::binary_search(m.bndPointSets[bi].begin(), m.bndPointSets[bi].end(), k.v[q]);
          if (all) bc = m.bndPointBc[bi];
        }
        if (bc == -100) {
          err = "boundary face without a boundary condition";
          return false;
        }
        boundary.push_back({pr.first, bc});
      } else {
        auto b = bndBc.find(k);
        if (b == bndBc.end()) {
          err = "boundary face without a boundary condition";
          return false;
        }
        boundary.push_back({pr.first, b->second});
      }
    }

  // Periodic pairing: centroid with each periodic coordinate folded onto the
  // low side of the domain, quantised to the periodic tolerance.
  std::vector<std::pair<Side, Side>> periodicPairs;
  std::vector<std::pair<Side, int>> realBnd;
  {
    double lo[3] = {1e300, 1e300, 1e300};
    for (int v = 0; v < m.nVerts; v++)
      for (int d = 0; d < nd; d++) lo[d] = std::min(lo[d], m.xv[(size_t)v * nd + d]);
    double hmin = 1e300;
    for (int d = 0; d < nd; d++) hmin = std::min(hmin, m.period[d] < 1e299 ? m.period[d] : 1e300);
    double q = std::max(m.periodicTol, 1e-9) * 10.0;
    std::map<std::array<long long, 3>, std::vector<std::pair<Side, int>>> buckets;
    for (auto &b : boundary) {
      if (b.second != PERIODIC) {
        realBnd.push_back(b);
        continue;
      }
      int nfv = nd == 2 ? 2 : 4;
      double c[3] = {0, 0, 0};
      for (int i = 0; i < nfv; i++) {
        int lv = nd == 2 ? kQuadFace[b.first.f][i] : kHexFace[b.first.f][i];
        int v = m.c2v[(size_t)b.first.e * m.nNodes + lv];
        for (int d = 0; d < nd; d++) c[d] += m.xv[(size_t)v * nd + d] / nfv;
      }
      std::array<long long, 3> key{0, 0, 0};
      for (int d = 0; d < nd; d++) {
        double x = c[d];
        if (m.period[d] < 1e299) {
          double r = (x - lo[d]) / m.period[d];
          double fl = std::floor(r + 1e-9);
          x -= fl * m.period[d];
          if (std::fabs(x - lo[d] - m.period[d]) < q) x = lo[d];
        }
        key[d] = std::llround(x / q);
      }
      buckets[key].push_back(b);
    }
    for (auto &kv : buckets) {
      auto &v = kv.second;
      if (v.size() != 2) {
        err = "Unmatched periodic faces exist.";
        return false;
      }
      periodicPairs.push_back({v[0].first, v[1].first});
    }
  }

  // Flux-point positions for orientation matching.
  auto fp = loc_fpts(nd, order, ptsType);
  std::vector<double> Nf(fp.size() * nN);
  for (size_t q = 0; q < fp.size(); q++) sf.eval(fp[q], &Nf[q * nN]);
  auto facePos = [&](int e, int f, std::vector<double> &out) {
    out.assign((size_t)nPF * 3, 0.0);
    const int *cv = &m.c2v[(size_t)e * nN];
    for (int j = 0; j < nPF; j++) {
      const double *N = &Nf[(size_t)(f * nPF + j) * nN];
      for (int d = 0; d < nd; d++) {
        double x = 0.0;
        for (int n = 0; n < nN; n++) x += N[n] * m.xv[(size_t)cv[n] * nd + d];
        out[(size_t)j * 3 + d] = x;
      }
    }
  };

  auto make_face = [&](Side a, Side b, bool periodic) -> bool {
    // Left side = smaller (element, local face): the reference's choice.
    if (b.e < a.e || (b.e == a.e && b.f < a.f)) std::swap(a, b);
    Face F;
    F.eL = a.e;
    F.locL = a.f;
    F.eR = b.e;
    F.locR = b.f;
    F.bc = BC_NONE;
    F.fptR.resize(nPF);
    std::vector<double> pl, pr;
    facePos(a.e, a.f, pl);
    facePos(b.e, b.f, pr);
    double shift[3] = {0, 0, 0};
    if (periodic) {
      double cl[3] = {0, 0, 0}, cr[3] = {0, 0, 0};
      for (int j = 0; j < nPF; j++)
        for (int d = 0; d < nd; d++) {
          cl[d] += pl[(size_t)j * 3 + d] / nPF;
          cr[d] += pr[(size_t)j * 3 + d] / nPF;
        }
      for (int d = 0; d < nd; d++) shift[d] = cl[d] - cr[d];
    }
    double scale = 0;
    for (int j = 0; j < nPF; j++)
      for (int d = 0; d < nd; d++) scale = std::max(scale, std::fabs(pl[(size_t)j * 3 + d] - pl[d]));
    if (scale == 0) scale = 1;
    for (int i = 0; i < nPF; i++) {
      int best = -1;
      double bd = 1e300;
      for (int j = 0; j < nPF; j++) {
        double dd = 0;
        for (int d = 0; d < nd; d++) {
          double t = pl[(size_t)i * 3 + d] - (pr[(size_t)j * 3 + d] + shift[d]);
          dd += t * t;
        }
        if (dd < bd) {
          bd = dd;
          best = j;
        }
      }
      if (nPF > 1 && std::sqrt(bd) > 1e-6 * scale + 1e-12) {
        err = "cannot orient face flux points";
        return false;
      }
      F.fptR[i] = b.f * nPF + best;
    }
    faces.push_back(std::move(F));
    return true;
  };

  for (auto &p : interior)
    if (!make_face(p.first, p.second, false)) return false;
  for (auto &p : periodicPairs)
    if (!make_face(p.first, p.second, true)) return false;
  for (auto &b : realBnd) {
    Face F;
    F.eL = b.first.e;
    F.locL = b.first.f;
    F.eR = -1;
    F.locR = -1;
    F.bc = b.second;
    faces.push_back(std::move(F));
  }
  return true;
}

bool build_geometry(const Mesh &m, int order, int ptsType, Geometry &g, std::string &err) {
  const int nd = m.nDims;
  auto sp = loc_spts(nd, order, ptsType);
  auto fp = loc_fpts(nd, order, ptsType);
  Operators op;  // only tNorm is needed here
  const int nS = (int)sp.size(), nF = (int)fp.size(), E = m.nEles;
  const int n1 = order + 1, nPF = nd == 2 ? n1 : n1 * n1;
  g.pos_spts.assign((size_t)nS * E * nd, 0.0);
  g.pos_fpts.assign((size_t)nF * E * nd, 0.0);
  g.detJac_spts.assign((size_t)nS * E, 0.0);
  g.detJac_fpts.assign((size_t)nF * E, 0.0);
  g.JGinv_spts.assign((size_t)nd * nS * E * nd, 0.0);
  g.norm_fpts.assign((size_t)nF * E * nd, 0.0);
  g.dA_fpts.assign((size_t)nF * E, 0.0);

  ShapeFn sf;
  if (!sf.init(nd, m.nNodes, err)) return false;
  const int nN = m.nNodes;
  std::vector<double> Ns((size_t)nS * nN), dNs((size_t)nS * nN * nd), Nf((size_t)nF * nN), dNf((size_t)nF * nN * nd);
  for (int s = 0; s < nS; s++) {
    sf.eval(sp[s], &Ns[(size_t)s * nN]);
    sf.deval(sp[s], &dNs[(size_t)s * nN * nd]);
  }
  for (int f = 0; f < nF; f++) {
    sf.eval(fp[f], &Nf[(size_t)f * nN]);
    sf.deval(fp[f], &dNf[(size_t)f * nN * nd]);
  }
  std::vector<std::array<double, 3>> X(nN);
  static const double tq[4][2] = {{0, -1}, {1, 0}, {0, 1}, {-1, 0}};
  static const double th[6][3] = {{0, 0, -1}, {0, 0, 1}, {-1, 0, 0}, {1, 0, 0}, {0, -1, 0}, {0, 1, 0}};

  for (int e = 0; e < E; e++) {
    for (int n = 0; n < m.nNodes; n++)
      for (int d = 0; d < nd; d++) X[n][d] = m.xv[(size_t)m.c2v[(size_t)e * m.nNodes + n] * nd + d];
    for (int s = 0; s < nS; s++) {
      double J[3][3] = {{0}};  // J[dref][dphys] = Jac_spts(dref, s, e, dphys)
      for (int d = 0; d < nd; d++) {
        double x = 0;
        for (int n = 0; n < m.nNodes; n++) x += Ns[(size_t)s * nN + n] * X[n][d];
        g.pos_spts[((size_t)s * E + e) * nd + d] = x;
      }
      for (int r = 0; r < nd; r++)
        for (int d = 0; d < nd; d++) {
          double v = 0;
          for (int n = 0; n < m.nNodes; n++) v += dNs[((size_t)s * nN + n) * nd + r] * X[n][d];
          J[r][d] = v;
        }
      double det;
      double A[3][3];
      if (nd == 2) {
        det = J[0][0] * J[1][1] - J[0][1] * J[1][0];
        A[0][0] = J[1][1];
        A[0][1] = -J[1][0];
        A[1][0] = -J[0][1];
        A[1][1] = J[0][0];
      } else {
        double xr = J[0][0], xs = J[1][0], xt = J[2][0];
        double yr = J[0][1], ys = J[1][1], yt = J[2][1];
        double zr = J[0][2], zs = J[1][2], zt = J[2][2];
        det = xr * (ys * zt - yt * zs) - xs * (yr * zt - yt * zr) + xt * (yr * zs - ys * zr);
        A[0][0] = ys * zt - yt * zs; A[0][1] = xt * zs - xs * zt; A[0][2] = xs * yt - xt * ys;
        A[1][0] = yt * zr - yr * zt; A[1][1] = xr * zt - xt * zr; A[1][2] = xt * yr - xr * yt;
        A[2][0] = yr * zs - ys * zr; A[2][1] = xs * zr - xr * zs; A[2][2] = xr * ys - xs * yr;
      }
      if (det < 0) {
        err = "Negative Jacobian at solution points.";  // reference: solver.cpp:1638
        return false;
      }
      g.detJac_spts[(size_t)s * E + e] = det;
      for (int a = 0; a < nd; a++)
        for (int b = 0; b < nd; b++) g.JGinv_spts[(((size_t)a * nS + s) * E + e) * nd + b] = A[a][b];
    }
    for (int f = 0; f < nF; f++) {
      double J[3][3] = {{0}};
      for (int d = 0; d < nd; d++) {
        double x = 0;
        for (int n = 0; n < m.nNodes; n++) x += Nf[(size_t)f * nN + n] * X[n][d];
        g.pos_fpts[((size_t)f * E + e) * nd + d] = x;
      }
      for (int r = 0; r < nd; r++)
        for (int d = 0; d < nd; d++) {
          double v = 0;
          for (int n = 0; n < m.nNodes; n++) v += dNf[((size_t)f * nN + n) * nd + r] * X[n][d];
          J[r][d] = v;
        }
      double det, A[3][3];
      if (nd == 2) {
        det = J[0][0] * J[1][1] - J[0][1] * J[1][0];
        A[0][0] = J[1][1];
        A[0][1] = -J[1][0];
        A[1][0] = -J[0][1];
        A[1][1] = J[0][0];
      } else {
        double xr = J[0][0], xs = J[1][0], xt = J[2][0];
        double yr = J[0][1], ys = J[1][1], yt = J[2][1];
        double zr = J[0][2], zs = J[1][2], zt = J[2][2];
        det = xr * (ys * zt - yt * zs) - xs * (yr * zt - yt * zr) + xt * (yr * zs - ys * zr);
        A[0][0] = ys * zt - yt * zs; A[0][1] = xt * zs - xs * zt; A[0][2] = xs * yt - xt * ys;
        A[1][0] = yt * zr - yr * zt; A[1][1] = xr * zt - xt * zr; A[1][2] = xt * yr - xr * yt;
        A[2][0] = yr * zs - ys * zr; A[2][1] = xs * zr - xr * zs; A[2][2] = xr * ys - xs * yr;
      }
      g.detJac_fpts[(size_t)f * E + e] = det;
      int iFace = f / nPF;
      const double *t = nd == 2 ? tq[iFace] : th[iFace];
      double nrm[3];
      for (int d1 = 0; d1 < nd; d1++) {
        nrm[d1] = 0.0;
        for (int d2 = 0; d2 < nd; d2++) nrm[d1] += A[d2][d1] * t[d2];
      }
      double dA = 0;
      for (int d = 0; d < nd; d++) dA += nrm[d] * nrm[d];
      dA = std::sqrt(dA);
      if (std::fabs(dA) < 1e-10) {
        dA = 0.0;
        for (int d = 0; d < nd; d++) nrm[d] = 0.0;
      } else {
        for (int d = 0; d < nd; d++) nrm[d] /= dA;
      }
      g.dA_fpts[(size_t)f * E + e] = dA;
      for (int d = 0; d < nd; d++) g.norm_fpts[((size_t)f * E + e) * nd + d] = nrm[d];
    }
  }
  (void)op;
  return true;
}

bool initial_condition(const Input &in, const Geometry &g, int nSpts, int nEles, int kind,
                       const double *prm, int nprm, std::vector<double> &U, std::string &err) {
  const int nd = in.nDims, nF = in.nFields, E = nEles;
  const double gam = in.gamma;
  const double PI = 3.141592653589793238462643383279502884;
  U.assign((size_t)nSpts * E * nF, 0.0);
  auto P = [&](int i, double def) { return (prm && i < nprm) ? prm[i] : def; };
  int deckIc = in.icType;
  for (int s = 0; s < nSpts; s++)
    for (int e = 0; e < E; e++) {
      const double *x = &g.pos_spts[((size_t)s * E + e) * nd];
      double X = x[0], Y = x[1], Z = nd == 3 ? x[2] : 0.0;
      double rho, u, v, w = 0.0, p;
      double *Ue = &U[((size_t)s * E + e) * nF];
      if (kind == IC_DECK && deckIc == 0) {
        // reference: src/ele.cpp:739-756
        rho = in.rhoIC;
        u = in.vxIC;
        v = in.vyIC;
        w = nd == 3 ? in.vzIC : 0.0;
        p = in.pIC;
        Ue[0] = rho;
        Ue[1] = rho * u;
        Ue[2] = rho * v;
        if (nd == 3) Ue[3] = rho * w;
        Ue[nd + 1] = p / (gam - 1) + (0.5 * rho * (u * u + v * v + w * w));
        continue;
      } else if (kind == IC_DECK && deckIc == 1) {
        // reference: src/ele.cpp:757-776 (+1e-5 in the exponent and the 1e-3
        // density clamp are the reference's)
        double eps = 5.0;
        double f = 1.0 - (X * X + Y * Y);
        rho = std::max(std::pow(1. - eps * eps * (gam - 1.) / (8. * gam * PI * PI) * std::exp(f),
                                1.0 / (gam - 1.0) + 1e-5),
                       1e-3);
        u = 1. - eps * Y / (2. * PI) * std::exp(f / 2.);
        v = 1. + eps * X / (2. * PI) * std::exp(f / 2.);
        p = std::pow(rho, gam);
        Ue[0] = rho;
        Ue[1] = rho * u;
        Ue[2] = rho * v;
        if (nd == 3) Ue[3] = 0.;
        Ue[nd + 1] = p / (gam - 1) + (0.5 * rho * (u * u + v * v));
        continue;
      } else if (kind == IC_DECK && deckIc == 2) {
        // reference: src/ele.cpp:777-801
        double eps = 1.0, rc = 1.0, Minf = .3, Uinf = 1, rhoInf = 1;
        double theta = in.vortexAngle;
        double Pinf = std::pow(Minf, -2) / gam;
        double eM = (eps * Minf) * (eps * Minf);
        double f = -(X * X + Y * Y) / (rc * rc);
        u = Uinf * (std::cos(theta) - Y * eps / rc * std::exp(f / 2.));
        v = Uinf * (std::sin(theta) + X * eps / rc * std::exp(f / 2.));
        rho = rhoInf * std::pow(1. - (gam - 1.) / 2. * eM * std::exp(f), gam / (gam - 1.0));
        p = Pinf * std::pow(1. - (gam - 1.) / 2. * eM * std::exp(f), gam / (gam - 1.0));
        Ue[0] = rho;
        Ue[1] = rho * u;
        Ue[2] = rho * v;
        if (nd == 3) Ue[3] = 0.;
        Ue[nd + 1] = p / (gam - 1) + (0.5 * rho * (u * u + v * v));
        continue;
      } else if (kind == IC_VORTEX) {
        double eps = P(0, 5.0), xc = P(1, 0.0), yc = P(2, 0.0), M = P(3, 0.5);
        double dx = X - xc, dy = Y - yc;
        double f = 1.0 - (dx * dx + dy * dy);
        rho = std::pow(1.0 - eps * eps * (gam - 1.0) / (8.0 * gam * PI * PI) * std::exp(f), 1.0 / (gam - 1.0));
        u = M * std::sqrt(gam) - eps * dy / (2.0 * PI) * std::exp(0.5 * f);
        v = eps * dx / (2.0 * PI) * std::exp(0.5 * f);
        p = std::pow(rho, gam);
      } else if (kind == IC_TGV) {
        double M = P(0, 0.1);
        double p0 = 1.0 / (gam * M * M);
        u = std::sin(X) * std::cos(Y) * std::cos(Z);
        v = -std::cos(X) * std::sin(Y) * std::cos(Z);
        w = 0.0;
        p = p0 + (std::cos(2.0 * X) + std::cos(2.0 * Y)) * (std::cos(2.0 * Z) + 2.0) / 16.0;
        rho = p / p0;
      } else if (kind == IC_UNIFORM) {
        rho = in.rhoBound;
        u = in.uBound;
        v = in.vBound;
        w = nd == 3 ? in.wBound : 0.0;
        p = in.pBound;
      } else {
        err = "unknown initial condition";
        return false;
      }
      Ue[0] = rho;
      Ue[1] = rho * u;
      Ue[2] = rho * v;
      if (nd == 3) Ue[3] = rho * w;
      Ue[nd + 1] = p / (gam - 1.0) + 0.5 * rho * (u * u + v * v + w * w);
    }
  return true;
}

}  // namespace fr
