// Host-side setup for the B200 Flux Reconstruction path: run-time options
// (the reference deck format), 1-D point sets and polynomials, dense FR
// operator matrices, mesh generation and connectivity, and metric terms.
//
// Everything here runs once per case at setup; the per-stage work is on the
// GPU (kernels/*.cu).  Array layouts follow the reference solver: row-major,
// last index fastest, state as [point][element][field]
// (reference: include/matrix.hpp:52-116, src/matrix.cpp:329-341).
#pragma once

#include <array>
#include <cstdint>
#include <string>
#include <vector>

namespace fr {

// Element types (reference: include/global.hpp:78-85).
enum EType { QUAD = 1, HEX = 4 };

// Boundary-condition codes (reference: include/global.hpp:116-132).
enum BcType {
  BC_NONE = -1,
  PERIODIC = 0,
  CHAR_INOUT = 1,
  SUP_IN = 2,
  SUP_OUT = 3,
  SUB_IN = 4,
  SUB_OUT = 5,
  SLIP_WALL = 8,
  ISOTHERMAL_NOSLIP = 9,
  ADIABATIC_NOSLIP = 10,
  SYMMETRY = 12,
  ISOTHERMAL_NOSLIP_MOVING = 13
};

// Point-set types for solution points ("spts_type_quad").
enum PtsType { PTS_LEGENDRE = 0, PTS_LOBATTO = 1, PTS_EQUIDISTANT = 2 };

int bc_from_string(const std::string &s);  // reference: src/global.cpp:43-58

// Run-time options on the residual/update path, with the reference's names,
// defaults and derived values (reference: src/input.cpp:257-523).
struct Input {
  int equation = 1;
  int icType = 0;
  int nDims = 2;
  int nFields = 4;
  double gamma = 1.4;
  double rhoBound = 1.0, uBound = 0.2, vBound = 0.0, wBound = 0.0,
         pBound = 0.7142857143;
  double rhoIC = 1.0, vxIC = 0.2, vyIC = 0.0, vzIC = 0.0, pIC = 0.7142857143;
  double vortexAngle = 0.4636476090008061;  // atan(0.5)
  double vortexXmin = -5, vortexXmax = 5, vortexYmin = -5, vortexYmax = 5;
  int errorNorm = 1, quadOrder = 10;  // error integrals against an exact solution (testCase 1)
  int timeType = 4;
  int dtType = 0;
  int iterMax = 0;
  double CFL = 0.0;
  double maxTime = 0.0;
  double dt = 0.0;
  int viscous = 0;
  int motion = 0;
  double moveAx = 0, moveAy = 0, moveFx = 0, moveFy = 0, moveAr = 0, moveFr = 0;
  int order = 3;
  int riemannType = 0;
  int testCase = 0;
  // viscous (LDG) parameters
  double penFact = 0.0, tau = 1.0;
  double Re = 0.0, Lref = 1.0, muGas = 1.827e-5, prandtl = 0.72, SGas = 120.0,
         TGas = 291.15, RGas = 286.9;
  int fixVis = 0;
  double TBound = 300.0, TWall = 300.0, MachBound = 0.0, nxBound = 1.0,
         nyBound = 0.0, nzBound = 0.0, MachWall = 0.0, nxWall = 1.0,
         nyWall = 0.0, nzWall = 0.0;
  double mu_inf = 0.0, rt_inf = 0.0, c_sth = 0.0, muBound = 0.0;
  // the viscous free-stream values are non-dimensional (done once, when the
  // deck is read, as input::readInputFile does; a Gmsh mesh read afterwards
  // finalises the inputs again for its nDims)
  bool nonDimensional = false;
  double uWall = 0.0, vWall = 0.0, wWall = 0.0;
  // mesh
  int meshType = 1;
  std::string meshFileName;
  int nx = 10, ny = 10, nz = 10;
  double xmin = -10, xmax = 10, ymin = -10, ymax = 10, zmin = -10, zmax = 10;
  std::string create_bcTop = "periodic", create_bcBottom = "periodic",
              create_bcLeft = "periodic", create_bcRight = "periodic",
              create_bcFront = "periodic", create_bcBack = "periodic";
  std::vector<std::pair<std::string, std::string>> meshBounds;  // mesh_bound
  double periodicDX = 1e300, periodicDY = 1e300, periodicDZ = 1e300;
  double periodicTol = 1e-6;
  int resType = 2;
  int sptsTypeQuad = PTS_LEGENDRE;
  int vcjhSchemeQuad = 0;
  int PMG = 0, lowOrder = 0, smoothSteps = 1;
  int restart = 0, restartIter = 0;
  // output (reference: src/input.cpp:428-433)
  std::string dataFileName = "simData";
  int plotType = 1, plotFreq = 100;
  // derived
  int nRKSteps = 4;
  std::vector<double> RKa, RKb;
};

// Reads a deck ("key value [comment]" lines; first match wins), applies the
// reference defaults and derived quantities.  Returns false with `err` set on
// a malformed file or an unsupported option value.
bool read_deck(const std::string &path, Input &in, std::string &err);
// Fills nFields, the RK tables and (viscous) the non-dimensional gas constants.
bool finalize_input(Input &in, std::string &err);

// --- points and polynomials (reference: src/points.cpp, src/polynomials.cpp)
std::vector<double> pts1d(int ptsType, int order);
std::vector<double> qwts1d(int order);  // Gauss-Legendre weights
double lagrange(const std::vector<double> &x, double y, int mode);
double dlagrange(const std::vector<double> &x, double y, int mode);
double legendre(double r, int n);
double dlegendre(double r, int n);
double compute_eta(int scheme, int order);
double dvcjh_1d(double r, int mode, int order, double eta);
double cfl_limit(int order);  // reference: src/global.cpp:81-105

struct Pt {
  double x = 0, y = 0, z = 0;
  double operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
std::vector<Pt> loc_spts(int nDims, int order, int ptsType);
std::vector<Pt> loc_fpts(int nDims, int order, int ptsType);
std::vector<double> spt_weights(int nDims, int order);   // getQptWeights
std::vector<double> face_weights(int nDims, int order);  // surface weights

// Dense FR operator matrices for one (element type, order), row-major.
struct Operators {
  int nDims = 0, order = 0, nSpts = 0, nFpts = 0;
  std::vector<double> ext;        // [nFpts][nSpts]   opp_spts_to_fpts
  std::vector<double> grad[3];    // [nSpts][nSpts]   opp_grad_spts[d]
  std::vector<double> extFn[3];   // [nFpts][nSpts]   opp_extrapolateFn[d]
  std::vector<double> corr;       // [nSpts][nFpts]   opp_correction
  std::vector<double> corrU[3];   // [nSpts][nFpts]   opp_correctU[d]
  int nSptsPro = 0, nSptsRes = 0;
  std::vector<double> prolong;    // [nSptsPro][nSpts]
  std::vector<double> restrict_;  // [nSptsRes][nSpts]
  std::vector<double> tNorm;      // [nFpts][nDims] reference-space face normal
};
void build_operators(int nDims, int order, int ptsType, int vcjh, Operators &op);

// --- mesh -------------------------------------------------------------------
// Quads or hexes of any geometric order the reference reads: Lagrange quads
// of (n+1)^2 nodes, Lagrange hexes of (n+1)^3 nodes and the 20-node
// serendipity hex, in Gmsh's node numbering (the first 4 or 8 are corners).
struct Mesh {
  int nDims = 2;
  int nVerts = 0;
  std::vector<double> xv;  // [nVerts][nDims]
  int nEles = 0;
  int nNodes = 4;
  std::vector<int> c2v;  // [nEles][nNodes]
  // Boundary faces given by their vertices (nDims==2: 2, 3: 4) and BC code.
  std::vector<std::array<int, 4>> bndFaceVerts;
  std::vector<int> bndFaceBc;
  double period[3] = {1e300, 1e300, 1e300};
  double periodicTol = 1e-6;
  // Alternatively, boundaries as vertex sets (Gmsh input): a boundary face
  // takes the BC of the first set holding all its vertices
  // (reference: src/geo.cpp:290-305, 476-497).
  std::vector<std::vector<int>> bndPointSets;  // sorted vertex ids per boundary
  std::vector<int> bndPointBc;
};

// Gmsh 2.x ASCII reader for quads (types 3, 10, 36-38, 47-51) and hexes
// (types 5, 12, 17, 92-94), with $PhysicalNames boundaries mapped through the
// deck's mesh_bound entries (reference: src/geo.cpp:1021-1475).  Triangles,
// tets and prisms (which the reference reads as collapsed quads and hexes) and
// meshes mixing node counts are refused.
bool read_gmsh(const std::string &path, Input &in, Mesh &m, std::string &err);

// Cartesian generator (reference: src/geo.cpp:1477-1762): same vertex and
// element numbering, BCs from the create_bc* options.
bool create_cartesian_mesh(const Input &in, Mesh &m, std::string &err);
// Moves interior vertices by U(-frac*h, frac*h) per coordinate from a seeded
// std::mt19937_64 (top 53 bits -> [0,1)), vertices in index order.
void perturb_interior_vertices(const Input &in, Mesh &m, uint64_t seed, double frac);

// One conforming face between two elements or on a boundary.
struct Face {
  int eL, locL;        // left element and its local face
  int eR, locR;        // right element / local face, -1 on a boundary
  int bc;              // BC code on a boundary face, else BC_NONE
  std::vector<int> fptR;  // right-element flux point for each left face point
};

// Face connectivity by hashing sorted vertex lists (O(n log n)); periodic
// boundary faces paired by their centroids modulo the period.  The left
// element of a face is the one with the smaller (element, local face) pair,
// which is the choice the reference makes (src/geo.cpp:509-566, 1764-1852).
bool build_faces(const Mesh &m, int order, int ptsType, std::vector<Face> &faces,
                 std::string &err);

// Metric terms at solution and flux points (reference: src/solver.cpp:165-317,
// 1587-1694), arrays in the reference layout.
struct Geometry {
  std::vector<double> pos_spts;     // [nSpts][nEles][nDims]
  std::vector<double> pos_fpts;     // [nFpts][nEles][nDims]
  std::vector<double> detJac_spts;  // [nSpts][nEles]
  std::vector<double> JGinv_spts;   // [nDims][nSpts][nEles][nDims]
  std::vector<double> norm_fpts;    // [nFpts][nEles][nDims]
  std::vector<double> dA_fpts;      // [nFpts][nEles]
  std::vector<double> detJac_fpts;  // [nFpts][nEles]
};
bool build_geometry(const Mesh &m, int order, int ptsType, Geometry &g, std::string &err);

// Partition of the elements into nparts by recursive coordinate bisection
// of their centroids (the reference uses METIS, src/geo.cpp:2380-2470), and
// the halo of one part: its elements (ascending global ids; local id = index
// here) and every point of a face cut by the partition as (peer part, slot
// fpt*nOwned + local element), ordered by face and point so that both sides
// of a cut list the same points in the same order (src/mpiFace.cpp:122-175).
bool partition_elements(const Mesh &m, int nparts, std::vector<int> &part, std::string &err);
bool halo_plan(const Mesh &m, const std::vector<Face> &faces, int nPF, const std::vector<int> &part, int rank,
               std::vector<int> &owned, std::vector<int> &peer, std::vector<long long> &slot, std::string &err);
// True when nNodes names a quad (nDims 2) or hex (nDims 3) shape above.
bool shape_supported(int nDims, int nNodes);
// Shape functions N [nPts][nNodes] and their reference-space derivatives
// dN [nPts][nNodes][nDims] at the points `loc`.
bool shape_tables(int nDims, int nNodes, const std::vector<Pt> &loc, std::vector<double> &N,
                  std::vector<double> &dN, std::string &err);
// Physical positions of reference-space points `loc` in every element,
// [point][element][nDims] (reference: src/solver.cpp:1248-1313, shape_ppts).
bool positions_at(const Mesh &m, const std::vector<Pt> &loc, std::vector<double> &pos, std::string &err);

// --- solution files (output.cpp) ---------------------------------------------
// Plot points: the (P+3)^d grid of -1, the solution points' 1-D set, +1
// (reference: src/points.cpp:164-196), and the interpolation from the
// solution points, [nPpts][nSpts] (src/operators.cpp:145-165).
std::vector<Pt> loc_ppts(int nDims, int order, int ptsType);
std::vector<double> spts_to_ppts(int nDims, int order, int ptsType);
// The reference's ParaView file from primitive variables at the plot points
// Vp [nPpts][E][nDims+2], their positions [nPpts][E][nDims] and, on a moving
// mesh, the grid velocity there (same layout; null on a static mesh).
bool write_paraview(const std::string &path, int nDims, int order, int E, double time, long long iter,
                    const double *Vp, const double *pos, const double *gridVel, std::string &err);
// The reference's CSV file: primitives at the solution then flux points.
bool write_csv(const std::string &path, int nDims, int nS, int nFp, int E, const double *U, const double *Ufpts,
               const double *posS, const double *posF, double gamma, std::string &err);
// State [nS][E][nF] of a case of order `order` from a ParaView restart file
// of any order (interpolated when the orders differ), with its TIME and
// ITER comments when present.
bool read_restart_vtu(const std::string &path, const Input &in, int order, int E, std::vector<double> &U,
                      double &time, bool &hasTime, long long &iter, bool &hasIter, std::string &err);

// Initial conditions.  kinds: 0 = reference icType of the deck
// (src/ele.cpp:733-832), 1 = vortex (eps, xc, yc, Mach), 2 = Taylor-Green
// (Mach), 3 = uniform boundary state.
enum IcKind { IC_DECK = 0, IC_VORTEX = 1, IC_TGV = 2, IC_UNIFORM = 3 };
bool initial_condition(const Input &in, const Geometry &g, int nSpts, int nEles,
                       int kind, const double *prm, int nprm, std::vector<double> &U,
                       std::string &err);

}  // namespace fr
