// ORACLE — TEST INFRASTRUCTURE ONLY.
//
// A CPU restatement of Free CFD's unstructured finite-volume residual path,
// used solely by tests/, by __graft_entry__.smoke() and by the cpu_baseline
// leg of bench.py as the checker.  Nothing in the freecfd_b200 product links,
// imports or calls this file.
//
// It follows the reference sources line by line (paths relative to the
// reference's src/), keeps its AoS objects, std::map stencils and per-face
// state caches, and is compiled with -ffp-contract=off so every double
// operation rounds once, as the reference's default x86-64 build does:
//   grid/grid_create_elements.cc  create_nodes_cells 27-182, create_faces 184-412,
//                                 create_boundary_ghosts 702-772, HaveNodes 977-986
//   grid/grid.cc                  areas_volumes 123-181
//   set_bcs.cc                    set_bcs 35-260
//   main.cc                       set_lengthScales 456-491
//   face_interpolation_weights.cc 32-138, interpolate/interpolate.cc 36-119,320-343
//   lsqr_grad_map.cc 32-99, gradient_maps.cc 39-78
//   variable/variable.h           face_calculate 134-147, cell_gradient 193-216
//   material/material.cc 108-153
//   navier_stokes/*               ns.cc, ns_limiters.cc, ns_assemble_linear_system.cc,
//                                 ns_apply_bcs.cc, ns_roe.cc, ns_ausm_plus_up.cc,
//                                 ns_vanleer.cc, ns_convective_face_flux.cc,
//                                 ns_diffusive_face_flux.cc, ns_set_bcs.cc
//   time_step.cc                  update_time_step 143-224
//   navier_stokes/ns_time_terms.cc cons2prim 26-56, time_terms 107-186
//
// Parity status: pinned.  The reference's own sources compile here against
// single-process stand-ins for MPI, PETSc, ParMETIS and CGNS (oracle/ref,
// `make ref`), and tests/test_reference_pin.py requires this restatement to
// reproduce that compiled reference's doubles bit for bit (mesh, geometry,
// LSQ weights, ghosts, gradients, limiters, residual, mdot, k-omega terms,
// time terms, time step) over every mesh family, flux and limiter; the
// golden vectors in tests/golden/ are the compiled reference's outputs.
// NavierStokes::update_boundaries is declared and called by the reference but
// its source file is absent; update_boundaries() below is
// a documented reconstruction (first-order ghost update, as at initialise).
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <limits>
#include <map>
#include <memory>
#include <set>
#include <string>
#include <vector>

#include "deck.hpp"

namespace orc {

// ---------------------------------------------------------------- Vec3D (vec3d/vec3d.cc:29-211)
struct Vec3 {
  double comp[3];
  Vec3(double x = 0., double y = 0., double z = 0.) { comp[0] = x; comp[1] = y; comp[2] = z; }
  double dot(const Vec3 &r) const { return (comp[0] * r.comp[0] + comp[1] * r.comp[1] + comp[2] * r.comp[2]); }
  Vec3 cross(const Vec3 &r) const {
    Vec3 t;
    t.comp[0] = comp[1] * r.comp[2] - comp[2] * r.comp[1];
    t.comp[1] = -comp[0] * r.comp[2] + comp[2] * r.comp[0];
    t.comp[2] = comp[0] * r.comp[1] - comp[1] * r.comp[0];
    return t;
  }
  Vec3 norm() const;
  Vec3 &operator=(double r) { comp[0] = r; comp[1] = r; comp[2] = r; return *this; }
  Vec3 &operator*=(double r) { comp[0] *= r; comp[1] *= r; comp[2] *= r; return *this; }
  Vec3 operator*(double r) const { return Vec3(comp[0] * r, comp[1] * r, comp[2] * r); }
  Vec3 &operator/=(double r) { comp[0] /= r; comp[1] /= r; comp[2] /= r; return *this; }
  Vec3 operator/(double r) const { return Vec3(comp[0] / r, comp[1] / r, comp[2] / r); }
  Vec3 &operator+=(const Vec3 &r) { comp[0] += r.comp[0]; comp[1] += r.comp[1]; comp[2] += r.comp[2]; return *this; }
  Vec3 &operator-=(const Vec3 &r) { comp[0] -= r.comp[0]; comp[1] -= r.comp[1]; comp[2] -= r.comp[2]; return *this; }
  double &operator[](int i) { return comp[i]; }
  double operator[](int i) const { return comp[i]; }
};
inline double fabs(const Vec3 &v) { return std::sqrt(v.comp[0] * v.comp[0] + v.comp[1] * v.comp[1] + v.comp[2] * v.comp[2]); }
inline Vec3 Vec3::norm() const { return (*this) / fabs(*this); }
inline Vec3 operator*(double l, const Vec3 &r) { return Vec3(l * r.comp[0], l * r.comp[1], l * r.comp[2]); }
inline Vec3 operator+(const Vec3 &l, const Vec3 &r) { return Vec3(l.comp[0] + r.comp[0], l.comp[1] + r.comp[1], l.comp[2] + r.comp[2]); }
inline Vec3 operator-(const Vec3 &l, const Vec3 &r) { return Vec3(l.comp[0] - r.comp[0], l.comp[1] - r.comp[1], l.comp[2] - r.comp[2]); }

// ---------------------------------------------------------------- scalar helpers
// The residual below is templated on its scalar type S so the same code gives
// the FP64 residual (S=double) and a complex-step derivative (S=CStep).
struct CStep {  // a + i*b with the complex-step rules (analytic extension, branches on real part)
  double re, im;
  CStep(double r = 0., double i = 0.) : re(r), im(i) {}
};
inline double re_(double x) { return x; }
inline double re_(const CStep &x) { return x.re; }
inline CStep operator+(CStep a, CStep b) { return {a.re + b.re, a.im + b.im}; }
inline CStep operator-(CStep a, CStep b) { return {a.re - b.re, a.im - b.im}; }
inline CStep operator-(CStep a) { return {-a.re, -a.im}; }
inline CStep operator*(CStep a, CStep b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
inline CStep operator/(CStep a, CStep b) {
  // h^2 terms vanish for h=1e-30; keep first-order form for stability
  double d = b.re;
  return {a.re / d, (a.im * b.re - a.re * b.im) / (d * d)};
}
inline CStep operator+(CStep a, double b) { return {a.re + b, a.im}; }
inline CStep operator+(double a, CStep b) { return {a + b.re, b.im}; }
inline CStep operator-(CStep a, double b) { return {a.re - b, a.im}; }
inline CStep operator-(double a, CStep b) { return {a - b.re, -b.im}; }
inline CStep operator*(CStep a, double b) { return {a.re * b, a.im * b}; }
inline CStep operator*(double a, CStep b) { return {a * b.re, a * b.im}; }
inline CStep operator/(CStep a, double b) { return {a.re / b, a.im / b}; }
inline CStep operator/(double a, CStep b) { return {a / b.re, -a * b.im / (b.re * b.re)}; }
inline CStep &operator+=(CStep &a, CStep b) { a = a + b; return a; }
inline CStep &operator-=(CStep &a, CStep b) { a = a - b; return a; }
inline CStep &operator*=(CStep &a, CStep b) { a = a * b; return a; }
inline bool operator<(CStep a, CStep b) { return a.re < b.re; }
inline bool operator>(CStep a, CStep b) { return a.re > b.re; }
inline bool operator<=(CStep a, CStep b) { return a.re <= b.re; }
inline bool operator>=(CStep a, CStep b) { return a.re >= b.re; }
inline bool operator<(CStep a, double b) { return a.re < b; }
inline bool operator>(CStep a, double b) { return a.re > b; }
inline bool operator<=(CStep a, double b) { return a.re <= b; }
inline bool operator>=(CStep a, double b) { return a.re >= b; }
inline bool operator!=(CStep a, double b) { return a.re != b; }
inline bool operator==(CStep a, double b) { return a.re == b; }
inline bool operator<(double a, CStep b) { return a < b.re; }
inline bool operator>(double a, CStep b) { return a > b.re; }
inline bool operator<=(double a, CStep b) { return a <= b.re; }
inline bool operator>=(double a, CStep b) { return a >= b.re; }
inline CStep sqrt(CStep a) { double s = std::sqrt(a.re); return {s, a.im / (2. * s)}; }
inline CStep fabs(CStep a) { return a.re < 0. ? -a : a; }
inline CStep pow(CStep a, double e) { double p = std::pow(a.re, e); return {p, e * std::pow(a.re, e - 1.) * a.im}; }
inline CStep tanh(CStep a) { double t = std::tanh(a.re); return {t, (1. - t * t) * a.im}; }
using std::pow;
using std::sqrt;
using std::tanh;
inline double fabs(double x) { return std::fabs(x); }

// std::max / std::min semantics (NaN handling matters for the limiters)
template <class A, class B>
inline A smax(const A &a, const B &b) { return (a < b) ? A(b) : a; }
template <class A, class B>
inline A smin(const A &a, const B &b) { return (b < a) ? A(b) : a; }

template <class S>
struct V3 {  // Vec3D arithmetic over S
  S c[3];
  V3() { c[0] = S(0.); c[1] = S(0.); c[2] = S(0.); }
  V3(S x, S y, S z) { c[0] = x; c[1] = y; c[2] = z; }
  explicit V3(const Vec3 &v) { c[0] = S(v.comp[0]); c[1] = S(v.comp[1]); c[2] = S(v.comp[2]); }
  S &operator[](int i) { return c[i]; }
  const S &operator[](int i) const { return c[i]; }
};
template <class S> inline S vdot(const V3<S> &a, const V3<S> &b) { return (a.c[0] * b.c[0] + a.c[1] * b.c[1] + a.c[2] * b.c[2]); }
template <class S> inline S vdot(const V3<S> &a, const Vec3 &b) { return (a.c[0] * b.comp[0] + a.c[1] * b.comp[1] + a.c[2] * b.comp[2]); }
template <class S> inline S vdot(const Vec3 &a, const V3<S> &b) { return (a.comp[0] * b.c[0] + a.comp[1] * b.c[1] + a.comp[2] * b.c[2]); }
template <class S> inline V3<S> vadd(const V3<S> &a, const V3<S> &b) { return V3<S>(a.c[0] + b.c[0], a.c[1] + b.c[1], a.c[2] + b.c[2]); }
template <class S> inline V3<S> vsub(const V3<S> &a, const V3<S> &b) { return V3<S>(a.c[0] - b.c[0], a.c[1] - b.c[1], a.c[2] - b.c[2]); }
template <class S, class T> inline V3<S> vscale(const T &l, const V3<S> &r) { return V3<S>(l * r.c[0], l * r.c[1], l * r.c[2]); }
template <class S> inline V3<S> vscale(const S &l, const Vec3 &r) { return V3<S>(l * r.comp[0], l * r.comp[1], l * r.comp[2]); }

// ---------------------------------------------------------------- constants (grid.h, bc.h, ns.h)
enum { INTERNAL_FACE = -1, UNASSIGNED_FACE = -2 };
enum { INTERNAL = 1, BOUNDARY_GHOST = 3 };
enum { SYMMETRY = 1, WALL = 2, INLET = 3, OUTLET = 4 };
enum { NONE = -1, NO_REVERSE = 1, DAMP_REVERSE = 2, VELOCITY = 3, MDOT = 4, SLIP = 5, STAGNATION = 6, FORCE_SUPERSONIC = 7 };
enum { FIXED_T = 1, FIXED_Q = 2, ADIABATIC = 3 };
enum { BC_RHO = 1, BC_P = 2, BC_T = 3, BC_STATE = 4, BC_V = 5 };
enum { VK = 1, BJ = 2, MINMOD = 3 };
enum { FIRST = 1, SECOND = 2 };
enum { ROE = 1, VAN_LEER = 2, AUSM_PLUS_UP = 3, SD_SLAU = 4, SW = 5 };
enum { CURVILINEAR = 1, LSQR = 2, GREENGAUSS = 3 };
enum { WTLI = 0, IDW = 1, SIMPLE = 2 };

// ---------------------------------------------------------------- grid records (grid/grid.h:90-129)
struct Node : Vec3 {
  std::vector<int> cells, faces;
};
struct Face {
  int bc = INTERNAL_FACE;
  bool symmetry = false;
  int parent = -1, neighbor = -1;
  Vec3 centroid, normal;
  std::map<int, double> average;
  double area = 0.;
  std::vector<int> nodes;
  double closest_wall_distance = 0., dissipation_factor = 0.;
};
struct Cell {
  int type = INTERNAL;
  int bc = -1;
  double volume = 0., lengthScale = 0., closest_wall_distance = 0.;
  Vec3 centroid;
  std::vector<int> nodes, faces, neighborCells;
  std::map<int, Vec3> gradMap;
  bool HaveNodes(int n, const int *list) const {  // grid_create_elements.cc:977-986
    for (int i = 0; i < n; ++i) {
      bool match = false;
      for (size_t j = 0; j < nodes.size(); ++j)
        if (list[i] == nodes[j]) { match = true; break; }
      if (!match) return false;
    }
    return true;
  }
};
struct BCregion {  // bc.h:54-63
  int type = 0;
  // set_bcs.cc creates BCregion without initialising specified/thermalType; the
  // reference reads indeterminate values there.  This restatement uses NONE.
  int kind = NONE, specified = NONE, thermalType = NONE;
  double area = 0., total_area = 0.;
  Vec3 areaVec;
};

// ---------------------------------------------------------------- material (material/material.cc)
struct Material {
  double Mw = 28.97, R = 0., gamma = 1.4, Pref = 0., Tref = 0.;
  bool sutherland = false, prandtl = false;
  double mu = 0., lambda = 0., sut_mu_ref = 0., sut_T_ref = 0., sut_S = 0., Pr = 0.7;
  template <class S> S rho(const S &p, const S &T) const { return (p + Pref) / (R * (T + Tref)); }
  template <class S> S pres(const S &rho_, const S &T) const { return rho_ * R * (T + Tref) - Pref; }
  template <class S> S temp(const S &p, const S &rho_) const { return (p + Pref) / (R * rho_) - Tref; }
  template <class S> S a(const S &p, const S &T) const { return sqrt(gamma * (p + Pref) / rho(p, T)); }
  template <class S> S viscosity(const S &T) const {
    if (!sutherland) return S(mu);
    return sut_mu_ref * pow((T + Tref) / sut_T_ref, 1.5) * (sut_T_ref + sut_S) / (T + Tref + sut_S);
  }
  double Cp() const { return gamma * R / (gamma - 1.); }  // ideal gas branch, material.cc:142-153
  template <class S> S therm_cond(const S &T) const {
    if (!prandtl) return S(lambda);
    return Cp() * viscosity(T) / Pr;
  }
};

// ---------------------------------------------------------------- per-face state caches (ns_state_cache.h:26-59)
template <class S>
struct CellState {
  S p, p_center, T, T_center, rho, a, H;
  double volume = 0.;
  V3<S> V, V_center, Vn;
  CellState() : p(0.), p_center(0.), T(0.), T_center(0.), rho(0.), a(0.), H(0.) {}
};
template <class S>
struct FaceState {
  int index = 0, parent = 0, neighbor = 0, bc = -1;
  S T, mu, lambda;
  V3<S> V, gradu, gradv, gradw, gradT;
  Vec3 normal, tangent1, tangent2, left2right;
  double area = 0.;
  FaceState() : T(0.), mu(0.), lambda(0.) {}
};

struct Grid {
  int dimension = 3, bcCount = 0;
  double lengthScale = 0., globalTotalVolume = 0.;
  int nodeCount = 0, cellCount = 0, faceCount = 0;
  std::vector<Node> node;
  std::vector<Face> face;
  std::vector<Cell> cell;
  std::vector<std::set<int>> bocoNodes;
  std::vector<int> face2bc;
  std::vector<int> boundaryFaceCount;
  Node &cellNode(int c, int n) { return node[cell[c].nodes[n]]; }
  Face &cellFace(int c, int f) { return face[cell[c].faces[f]]; }
  Node &faceNode(int f, int n) { return node[face[f].nodes[n]]; }
};

struct Oracle {
  InputFile input;
  InputFile matfile;
  Grid grid;
  std::vector<BCregion> bc;
  Material material;
  // NavierStokes options (ns.cc:33-102)
  int order = SECOND, limiter_function = VK, flux = AUSM_PLUS_UP;
  double limiter_threshold = 0., Minf = 1.;
  double wdiss = 0.3, bl_height = 0.;  // ns.cc:76-77
  Vec3 moment_center;                  // writeoutput -> momentcenter (main.cc:240)
  int hex_method = LSQR, prism_method = LSQR, other_method = LSQR;
  int interp_method = WTLI, stencil_size = 2;
  // Variable<TYPE>::fixedonBC / bcValue for the NS variables (ns_set_bcs.cc)
  std::vector<char> p_fixed, T_fixed, rho_fixed, V_fixed, qdot_fixed, mdot_fixed, pt_fixed, Tt_fixed;
  std::vector<double> p_bc, T_bc, rho_bc, qdot_bc, mdot_bc, pt_bc, Tt_bc;
  std::vector<Vec3> V_bc;
  // Ghost-update reconstruction switch (see update_boundaries)
  int ghost_mode = 0;  // 0: first order (zero gradients), as at initialise; 1: face-centre BC state
  // Time stepping (time_step.cc)
  double cfl_max = 1000., cfl_local = 1000.;
  bool has_cfl_max = false, has_cfl_local = false;
  // RANS k-omega (rans.cc, rans_set_bcs.cc): options and fixed BC values
  bool turbulent = false;
  double kLow = 1e-10, kHigh = 1e8, omegaLow = 1e-2, ratioLimit = 1e8, Pr_t = 0.9;
  std::vector<char> kw_fixed, mut_fixed;
  std::vector<double> k_bc, omega_bc, mut_bc;
  std::string error;
};

// rans.cc:43-49 (model=k-omega: blending = 1 everywhere)
struct KOmega {
  static constexpr double sigma_k = 0.85, sigma_omega = 0.5, beta = 0.075, beta_star = 0.09, alpha = 5. / 9.;
};

// ================================================================ grid setup

// grid_create_elements.cc:27-182 (single partition: every cell is owned by rank 0)
static void create_nodes_cells(Grid &g, const double *xyz, int n_nodes, int n_cells, const int *cidx, const int *conn,
                               std::map<int, int> *g2l_out = nullptr) {
  std::map<int, int> nodeGlobal2Local;
  g.cell.reserve(n_cells);
  g.nodeCount = 0;
  for (int c = 0; c < n_cells; ++c) {
    int cellNodeCount = cidx[c + 1] - cidx[c];
    std::vector<int> cellNodes(cellNodeCount);
    for (int n = 0; n < cellNodeCount; ++n) {
      int ngid = conn[cidx[c] + n];
      if (nodeGlobal2Local.find(ngid) == nodeGlobal2Local.end()) {
        Node t;
        t.comp[0] = xyz[3 * ngid + 0]; t.comp[1] = xyz[3 * ngid + 1]; t.comp[2] = xyz[3 * ngid + 2];
        nodeGlobal2Local[ngid] = g.nodeCount;
        g.node.push_back(t);
        ++g.nodeCount;
      }
      cellNodes[n] = nodeGlobal2Local[ngid];
    }
    Cell t;
    t.type = INTERNAL;
    t.bc = -1;
    switch (cellNodeCount) {
      case 4: t.faces.assign(4, -1); break;
      case 5: t.faces.assign(5, -1); break;
      case 6: t.faces.assign(5, -1); break;
      case 8: t.faces.assign(6, -1); break;
      default: throw DeckError("unsupported element with " + std::to_string(cellNodeCount) + " nodes");
    }
    t.nodes = cellNodes;
    g.cell.push_back(t);
  }
  g.cellCount = (int)g.cell.size();
  (void)n_nodes;
  // node -> cells (114-129)
  for (int c = 0; c < g.cellCount; ++c) {
    for (size_t cn = 0; cn < g.cell[c].nodes.size(); ++cn) {
      int n = g.cell[c].nodes[cn];
      bool flag = false;
      for (size_t i = 0; i < g.node[n].cells.size(); ++i)
        if (g.node[n].cells[i] == c) { flag = true; break; }
      if (!flag) g.node[n].cells.push_back(c);
    }
  }
  // cell -> node neighbours (131-147)
  for (int c = 0; c < g.cellCount; ++c) {
    for (size_t cn = 0; cn < g.cell[c].nodes.size(); ++cn) {
      int n = g.cell[c].nodes[cn];
      for (size_t nc = 0; nc < g.node[n].cells.size(); ++nc) {
        int c2 = g.node[n].cells[nc];
        bool flag = false;
        for (size_t cc = 0; cc < g.cell[c].neighborCells.size(); ++cc)
          if (g.cell[c].neighborCells[cc] == c2) { flag = true; break; }
        if (!flag) g.cell[c].neighborCells.push_back(c2);
      }
    }
  }
  // boco node sets to local ids (151-162): identity here (all nodes are local, in first-seen order)
  for (auto &s : g.bocoNodes) {
    std::set<int> t;
    for (int id : s) {
      auto it = nodeGlobal2Local.find(id);
      if (it != nodeGlobal2Local.end()) t.insert(it->second);
    }
    s.swap(t);
  }
  if (g2l_out) g2l_out->swap(nodeGlobal2Local);
}

// grid_create_elements.cc:184-412
static void create_faces(Grid &g) {
  static const int hexaFaces[6][4] = {{0, 3, 2, 1}, {4, 5, 6, 7}, {1, 2, 6, 5}, {0, 4, 7, 3}, {1, 5, 4, 0}, {2, 3, 7, 6}};
  static const int prismFaces[5][4] = {{0, 2, 1, 0}, {3, 4, 5, 0}, {0, 3, 5, 2}, {1, 2, 5, 4}, {0, 1, 4, 3}};
  static const int pyraFaces[5][4] = {{0, 3, 2, 1}, {0, 1, 4, 0}, {1, 2, 4, 0}, {3, 4, 2, 0}, {0, 4, 3, 0}};
  static const int tetraFaces[4][3] = {{0, 2, 1}, {1, 2, 3}, {0, 3, 2}, {0, 1, 3}};
  g.faceCount = 0;
  for (int c = 0; c < g.cellCount; ++c) {
    int degenerate_face_count = 0;
    for (size_t cf = 0; cf < g.cell[c].faces.size(); ++cf) {
      bool degenerate = false;
      Face tf;
      int nn = 0;
      switch (g.cell[c].nodes.size()) {
        case 4: nn = 3; break;
        case 5: nn = (cf < 1) ? 4 : 3; break;
        case 6: nn = (cf < 2) ? 3 : 4; break;
        case 8: nn = 4; break;
      }
      tf.nodes.resize(nn);
      int tmp[4];
      tf.parent = c;
      tf.bc = INTERNAL_FACE;
      for (int fn = 0; fn < nn; ++fn) {
        switch (g.cell[c].nodes.size()) {
          case 4: tmp[fn] = g.cell[c].nodes[tetraFaces[cf][fn]]; break;
          case 5: tmp[fn] = g.cell[c].nodes[pyraFaces[cf][fn]]; break;
          case 6: tmp[fn] = g.cell[c].nodes[prismFaces[cf][fn]]; break;
          case 8: tmp[fn] = g.cell[c].nodes[hexaFaces[cf][fn]]; break;
        }
      }
      std::vector<int> unique_nodes;
      for (int fn = 0; fn < nn; ++fn) {
        bool skip = false;
        for (int i = 0; i < fn; ++i)
          if (tmp[fn] == tmp[i]) { skip = true; break; }
        if (!skip) unique_nodes.push_back(tmp[fn]);
      }
      if ((int)unique_nodes.size() != nn) {
        if (unique_nodes.size() == 2) { degenerate = true; degenerate_face_count++; }
        tf.nodes.resize(unique_nodes.size());
        nn = (int)unique_nodes.size();
        for (int fn = 0; fn < nn; ++fn) tmp[fn] = unique_nodes[fn];
      }
      bool internal = false, unique = true;
      tf.neighbor = -1;
      const Node &n0 = g.node[tmp[0]];
      for (size_t nc = 0; nc < n0.cells.size(); ++nc) {
        int i = n0.cells[nc];
        if (i != c && i < g.cellCount && g.cell[i].HaveNodes(nn, tmp)) {
          if (i > c) { tf.neighbor = i; internal = true; }
          else unique = false;
        }
      }
      if (unique && !degenerate) {
        for (int fn = 0; fn < nn; ++fn) tf.nodes[fn] = tmp[fn];
        if (!internal) {
          tf.bc = UNASSIGNED_FACE;
          std::vector<int> face_matched_bcs;
          int cell_matched_bc = -1;
          for (size_t nbc = 0; nbc < g.bocoNodes.size(); ++nbc) {
            bool match = true;
            for (int i = 0; i < nn; ++i)
              if (g.bocoNodes[nbc].find(tmp[i]) == g.bocoNodes[nbc].end()) { match = false; break; }
            if (match) face_matched_bcs.push_back((int)nbc);
            if (cell_matched_bc == -1) {
              match = true;
              for (size_t i = 0; i < g.cell[c].nodes.size(); ++i)
                if (g.bocoNodes[nbc].find(g.cell[c].nodes[i]) == g.bocoNodes[nbc].end()) { match = false; break; }
              if (match) cell_matched_bc = (int)nbc;
            }
          }
          if (face_matched_bcs.size() > 1) {
            for (size_t fbc = 0; fbc < face_matched_bcs.size(); ++fbc)
              if (face_matched_bcs[fbc] != cell_matched_bc) { tf.bc = face_matched_bcs[fbc]; break; }
          } else if (face_matched_bcs.size() == 1) {
            tf.bc = face_matched_bcs[0];
          }
        }
        for (size_t i = 0; i < g.cell[c].faces.size(); ++i)
          if (g.cell[c].faces[i] < 0) { g.cell[c].faces[i] = (int)g.face.size(); break; }
        if (internal) {
          for (size_t i = 0; i < g.cell[tf.neighbor].faces.size(); ++i)
            if (g.cell[tf.neighbor].faces[i] < 0) { g.cell[tf.neighbor].faces[i] = (int)g.face.size(); break; }
        }
        g.face.push_back(tf);
        ++g.faceCount;
      }
    }
    g.cell[c].faces.resize(g.cell[c].faces.size() - degenerate_face_count);
  }
  for (int f = 0; f < g.faceCount; ++f) {
    for (size_t n = 0; n < g.face[f].nodes.size(); ++n) g.faceNode(f, (int)n).faces.push_back(f);
    g.face[f].symmetry = false;
  }
}

// ---------------------------------------------------------------- face-based (Tecplot) grids

// grid_reader_tec.cc:36-278: Grid::readTEC.  Stream semantics kept: header
// lines up to the first line starting (after blanks) with a digit or '-',
// split at ',' then '=' (StringExplode, inputs.cc:363-376); block-packed
// coordinates; one optional comment line before each later block; 1-based
// indices.  Boundary zones: header lines read while the next line is not
// numeric (the grabbed ZONE line is processed after that test), ZONET names a
// new region, Nodes its node count; every zone node goes to the region of the
// last ZONET as the nearest boundary-face node (kd_nearest3; here an exact
// coordinate match, else the nearest, lowest id among equals).  Cell node
// lists: the sorted node set of each cell's faces (the reference's last face
// reads one index past faceConnIndex, grid_reader_tec.cc:240-243; for closed
// cells its nodes are in the set through the cell's other faces).
struct TecRaw {
  int nNodes = 0, nCells = 0, nFaces = 0;
  std::vector<double> xyz;
  std::vector<int> faceNodeCount, faceConnIndex, faceConnectivity, left, right;
  std::vector<std::set<int>> bocoNodes;
  std::vector<int> cellConnIndex, cellConnectivity;
};

static bool tec_first_numeric(std::istream &f) {
  while (std::isspace(f.peek())) f.get();
  int c = f.peek();
  return c == '-' || (c >= '0' && c <= '9');
}
static std::string tec_strip(const std::string &s) {
  std::string o;
  for (char c : s) if (!std::isspace((unsigned char)c)) o.push_back(c);
  return o;
}
static void tec_explode(std::string str, const std::string &sep, std::vector<std::string> *out) {
  size_t found = str.find_first_of(sep);
  while (found != std::string::npos) {
    if (found > 0) out->push_back(str.substr(0, found));
    str = str.substr(found + 1);
    found = str.find_first_of(sep);
  }
  if (str.length() > 0) out->push_back(str);
}

static TecRaw read_tec(const std::string &fileName) {
  TecRaw raw;
  std::ifstream file(fileName.c_str(), std::ios::in | std::ios::binary);
  if (!file.is_open()) throw DeckError("grid file " + fileName + " could not be found");
  std::string line;
  while (true) {
    if (tec_first_numeric(file)) break;
    if (!std::getline(file, line)) throw DeckError("error reading grid file " + fileName);
    line = tec_strip(line);
    std::vector<std::string> expression;
    tec_explode(line, ",", &expression);
    for (size_t i = 0; i < expression.size(); ++i) {
      std::vector<std::string> temp;
      tec_explode(expression[i], "=", &temp);
      if (temp.size() != 2) continue;
      if (temp[0] == "Nodes") raw.nNodes = std::atoi(temp[1].c_str());
      else if (temp[0] == "Elements") raw.nCells = std::atoi(temp[1].c_str());
      else if (temp[0] == "Faces") raw.nFaces = std::atoi(temp[1].c_str());
      else if (temp[0] == "ZONETYPE" && temp[1] != "FEPolyhedron") throw DeckError("ZONETYPE=" + temp[1] + " is not supported");
      else if (temp[0] == "DATAPACKING" && temp[1] != "BLOCK") throw DeckError("DATAPACKING=" + temp[1] + " is not supported");
      else if (temp[0] == "NumConnectedBoundaryFaces" && std::atoi(temp[1].c_str()) != 0) throw DeckError("NumConnectedBoundaryFaces>0");
      else if (temp[0] == "TotalNumBoundaryConnections" && std::atoi(temp[1].c_str()) != 0) throw DeckError("TotalNumBoundaryConnections>0");
    }
  }
  raw.xyz.assign(3 * (size_t)raw.nNodes, 0.);
  for (int i = 0; i < 3; ++i) for (int n = 0; n < raw.nNodes; ++n) file >> raw.xyz[3 * (size_t)n + i];
  if (!tec_first_numeric(file)) std::getline(file, line);
  raw.faceNodeCount.resize(raw.nFaces);
  raw.faceConnIndex.resize(raw.nFaces);
  int size = 0;
  for (int f = 0; f < raw.nFaces; ++f) {
    file >> raw.faceNodeCount[f];
    raw.faceConnIndex[f] = size;
    size += raw.faceNodeCount[f];
  }
  if (!tec_first_numeric(file)) std::getline(file, line);
  raw.faceConnectivity.resize(size);
  for (int i = 0; i < size; ++i) { file >> raw.faceConnectivity[i]; raw.faceConnectivity[i]--; }
  if (!tec_first_numeric(file)) std::getline(file, line);
  raw.left.resize(raw.nFaces);
  for (int f = 0; f < raw.nFaces; ++f) file >> raw.left[f];
  if (!tec_first_numeric(file)) std::getline(file, line);
  raw.right.resize(raw.nFaces);
  for (int f = 0; f < raw.nFaces; ++f) file >> raw.right[f];
  for (int f = 0; f < raw.nFaces; ++f) { raw.right[f]--; raw.left[f]--; }
  if (!file.good()) throw DeckError("grid file " + fileName + " is truncated");
  // boundary-face nodes (the kd-tree contents)
  std::vector<int> bnodes;
  {
    std::set<int> s;
    for (int f = 0; f < raw.nFaces; ++f)
      if (raw.right[f] < 0 || raw.left[f] < 0)
        for (int k = 0; k < raw.faceNodeCount[f]; ++k) s.insert(raw.faceConnectivity[raw.faceConnIndex[f] + k]);
    bnodes.assign(s.begin(), s.end());
  }
  auto nearest = [&](const double *q) {
    int best = -1;
    double bd = INFINITY;
    for (int n : bnodes) {
      const double *x = &raw.xyz[3 * (size_t)n];
      if (x[0] == q[0] && x[1] == q[1] && x[2] == q[2]) return n;
      double d = (x[0] - q[0]) * (x[0] - q[0]) + (x[1] - q[1]) * (x[1] - q[1]) + (x[2] - q[2]) * (x[2] - q[2]);
      if (d < bd) { bd = d; best = n; }
    }
    return best;
  };
  int bc_count = 0;
  bool line_grabbed = false;
  while (true) {
    int bcNodeCount = 0;
    while (true) {
      if (tec_first_numeric(file)) break;
      if (!line_grabbed) {
        if (!std::getline(file, line)) throw DeckError("error reading grid file " + fileName);
      }
      line_grabbed = false;
      line = tec_strip(line);
      std::vector<std::string> expression;
      tec_explode(line, ",", &expression);
      for (size_t i = 0; i < expression.size(); ++i) {
        std::vector<std::string> temp;
        tec_explode(expression[i], "=", &temp);
        if (temp.size() != 2) continue;
        if (temp[0] == "ZONET") bc_count++;
        else if (temp[0] == "Nodes") bcNodeCount = std::atoi(temp[1].c_str());
      }
    }
    if (bc_count == 0) throw DeckError("grid file: boundary zone without ZONE T=");
    std::vector<double> bcnodes(3 * (size_t)bcNodeCount);
    for (int i = 0; i < 3; ++i) for (int n = 0; n < bcNodeCount; ++n) file >> bcnodes[3 * (size_t)n + i];
    raw.bocoNodes.resize(bc_count);
    for (int n = 0; n < bcNodeCount; ++n) {
      int id = nearest(&bcnodes[3 * (size_t)n]);
      if (id >= 0) raw.bocoNodes[bc_count - 1].insert(id);
    }
    while (true) {
      std::getline(file, line);
      line = tec_strip(line);
      line_grabbed = true;
      if (line.substr(0, 4) == "ZONE") break;
      if (file.eof()) break;
    }
    if (file.eof()) break;
  }
  std::vector<std::set<int>> cellnodes(raw.nCells);
  for (int f = 0; f < raw.nFaces; ++f)
    for (int k = 0; k < raw.faceNodeCount[f]; ++k) {
      int n = raw.faceConnectivity[raw.faceConnIndex[f] + k];
      if (raw.left[f] >= 0) cellnodes[raw.left[f]].insert(n);
      if (raw.right[f] >= 0) cellnodes[raw.right[f]].insert(n);
    }
  raw.cellConnIndex.assign(raw.nCells + 1, 0);
  for (int c = 0; c < raw.nCells; ++c) {
    raw.cellConnIndex[c + 1] = raw.cellConnIndex[c] + (int)cellnodes[c].size();
    raw.cellConnectivity.insert(raw.cellConnectivity.end(), cellnodes[c].begin(), cellnodes[c].end());
  }
  return raw;
}

// grid_create_elements.cc:444-553: faces in file order, parent = left,
// neighbour = right, boundary regions from the node sets.  Each cell's face
// list is its faces in file order (the reference pads the list with one zero
// per face first, grid_create_elements.cc:107-121, which adds face 0 to every
// cell's face loops; not restated).
static void create_faces2(Grid &g, const TecRaw &raw, const std::map<int, int> &g2l) {
  for (int c = 0; c < g.cellCount; ++c) g.cell[c].faces.clear();
  g.faceCount = 0;
  for (int f = 0; f < raw.nFaces; ++f) {
    int parent = raw.left[f], neighbor = raw.right[f];
    if (parent < 0) throw DeckError("face without a left element");
    Face tf;
    tf.bc = (neighbor < 0) ? UNASSIGNED_FACE : INTERNAL_FACE;
    tf.parent = parent;
    tf.neighbor = neighbor;
    tf.nodes.resize(raw.faceNodeCount[f]);
    for (size_t fn = 0; fn < tf.nodes.size(); ++fn) tf.nodes[fn] = g2l.at(raw.faceConnectivity[raw.faceConnIndex[f] + fn]);
    if (tf.bc == UNASSIGNED_FACE) {
      std::vector<int> face_matched_bcs;
      int cell_matched_bc = -1;
      for (size_t nbc = 0; nbc < g.bocoNodes.size(); ++nbc) {
        bool match = true;
        for (size_t i = 0; i < tf.nodes.size(); ++i)
          if (g.bocoNodes[nbc].find(tf.nodes[i]) == g.bocoNodes[nbc].end()) { match = false; break; }
        if (match) face_matched_bcs.push_back((int)nbc);
        if (cell_matched_bc == -1) {
          match = true;
          for (size_t i = 0; i < g.cell[tf.parent].nodes.size(); ++i)
            if (g.bocoNodes[nbc].find(g.cell[tf.parent].nodes[i]) == g.bocoNodes[nbc].end()) { match = false; break; }
          if (match) cell_matched_bc = (int)nbc;
        }
      }
      if (face_matched_bcs.size() > 1) {
        for (size_t fbc = 0; fbc < face_matched_bcs.size(); ++fbc)
          if (face_matched_bcs[fbc] != cell_matched_bc) { tf.bc = face_matched_bcs[fbc]; break; }
      } else if (face_matched_bcs.size() == 1) {
        tf.bc = face_matched_bcs[0];
      } else {
        throw DeckError("couldn't find BC for face " + std::to_string(f));
      }
    }
    g.cell[tf.parent].faces.push_back((int)g.face.size());
    if (tf.bc == INTERNAL_FACE) g.cell[tf.neighbor].faces.push_back((int)g.face.size());
    g.face.push_back(tf);
    ++g.faceCount;
  }
  for (int f = 0; f < g.faceCount; ++f) {
    for (size_t n = 0; n < g.face[f].nodes.size(); ++n) g.faceNode(f, (int)n).faces.push_back(f);
    g.face[f].symmetry = false;
  }
}

// grid.cc:123-181
static void areas_volumes(Grid &g) {
  for (int f = 0; f < g.faceCount; ++f) {
    Face &F = g.face[f];
    if (F.nodes.size() == 4) {
      Vec3 d1 = g.faceNode(f, 2) - g.faceNode(f, 0);
      Vec3 d2 = g.faceNode(f, 3) - g.faceNode(f, 1);
      F.normal = d1.cross(d2);
      F.area = 0.5 * fabs(F.normal);
      F.normal = F.normal.norm();
    } else {
      Vec3 areaVec;
      areaVec = 0.;
      Vec3 centroid = g.faceNode(f, 0);
      for (size_t n = 1; n < F.nodes.size(); ++n) {
        size_t next = n + 1;
        if (next == F.nodes.size()) next = 0;
        Vec3 patchArea = 0.5 * (Vec3(g.faceNode(f, (int)n)) - centroid).cross(Vec3(g.faceNode(f, (int)next)) - centroid);
        areaVec += patchArea;
      }
      F.area = fabs(areaVec);
      F.normal = areaVec.norm();
    }
    F.centroid = 0.;
    for (size_t n = 0; n < F.nodes.size(); ++n) F.centroid += g.faceNode(f, (int)n);
    F.centroid /= double(F.nodes.size());
  }
  double totalVolume = 0.;
  for (int c = 0; c < g.cellCount; ++c) {
    Cell &C = g.cell[c];
    C.centroid = 0.;
    for (size_t cn = 0; cn < C.nodes.size(); ++cn) C.centroid += g.cellNode(c, (int)cn);
    C.centroid /= double(C.nodes.size());
    C.volume = 0.;
    for (size_t cf = 0; cf < C.faces.size(); ++cf) {
      int f = C.faces[cf];
      Vec3 base_area = g.face[f].area * g.face[f].normal;
      if (g.face[f].parent == c) base_area *= -1.;
      Vec3 base_area_norm = base_area.norm();
      Vec3 height = (C.centroid - g.face[f].centroid).dot(base_area_norm) * base_area_norm;
      C.volume += base_area.dot(height) / 3.;
    }
    totalVolume += C.volume;
  }
  g.globalTotalVolume = totalVolume;
}

// grid_create_elements.cc:702-772
static void create_boundary_ghosts(Grid &g) {
  std::vector<int> begin(g.bcCount);
  for (int b = 0; b < g.bcCount; ++b) {
    begin[b] = (int)g.cell.size();
    for (int f = 0; f < g.faceCount; ++f) {
      if (g.face[f].bc == b) {
        int parent = g.face[f].parent;
        Cell t;
        t.type = BOUNDARY_GHOST;
        t.bc = b;
        t.volume = g.cell[parent].volume;
        t.lengthScale = g.cell[parent].lengthScale;  // copied before set_lengthScales runs (reference order)
        t.closest_wall_distance = 0.;
        t.centroid = g.cell[parent].centroid + 2. * (g.face[f].centroid - g.cell[parent].centroid).dot(g.face[f].normal) * g.face[f].normal;
        g.face[f].neighbor = (int)g.cell.size();
        for (size_t fn = 0; fn < g.face[f].nodes.size(); ++fn) g.faceNode(f, (int)fn).cells.push_back(g.face[f].neighbor);
        g.cell.push_back(t);
      }
    }
  }
  int first_ghost = g.bcCount > 0 ? begin[0] : (int)g.cell.size();
  for (int c = 0; c < g.cellCount; ++c) {
    for (size_t cn = 0; cn < g.cell[c].nodes.size(); ++cn) {
      int n = g.cell[c].nodes[cn];
      for (size_t ng = 0; ng < g.node[n].cells.size(); ++ng) {
        int gh = g.node[n].cells[ng];
        if (gh >= first_ghost) {
          bool flag = false;
          for (size_t cg = 0; cg < g.cell[c].neighborCells.size(); ++cg)
            if (g.cell[c].neighborCells[cg] == gh) { flag = true; break; }
          if (!flag) {
            g.cell[c].neighborCells.push_back(gh);
            g.cell[gh].neighborCells.push_back(c);
          }
        }
      }
    }
  }
}

static bool withinBox(const Vec3 &p, const V3d &c1, const V3d &c2) {  // utilities.cc:37-49
  for (int i = 0; i < 3; ++i) {
    if (c1.c[i] > c2.c[i]) {
      if (p[i] > c1.c[i]) return false;
      if (p[i] < c2.c[i]) return false;
    } else {
      if (p[i] < c1.c[i]) return false;
      if (p[i] > c2.c[i]) return false;
    }
  }
  return true;
}

// set_bcs.cc:35-260
static void set_bcs_global(Oracle &O) {
  Grid &g = O.grid;
  Section &gs = O.input.section("grid", 0);
  int count = gs.sub("BC", 0).count;
  g.bcCount = count;
  g.face2bc.assign(g.faceCount, 0);
  std::vector<int> bc_counter(count, 0);
  for (int b = 0; b < count; ++b) {
    Subsection &region = gs.sub("BC", b);
    std::string pick = region.gs("pick").value;
    int pick_from = 0;
    if (pick.substr(0, 2) == "BC") { pick_from = std::atoi(pick.substr(2).c_str()); pick = "BC"; }
    if (region.gs("region").value == "box") {
      for (int f = 0; f < g.faceCount; ++f) {
        if ((g.face[f].bc >= 0 || g.face[f].bc == UNASSIGNED_FACE) &&
            withinBox(g.face[f].centroid, region.gv("corner_1").value, region.gv("corner_2").value)) {
          if (pick == "override") g.face[f].bc = b;
          else if (pick == "unassigned" && g.face[f].bc == UNASSIGNED_FACE) g.face[f].bc = b;
          else if (pick == "BC" && g.face[f].bc == (pick_from - 1)) g.face[f].bc = b;
        }
      }
    }
    BCregion r;
    std::string type = region.gs("type").value, kind = region.gs("kind").value;
    if (type == "wall") r.type = WALL;
    if (type == "inlet") r.type = INLET;
    if (type == "outlet") r.type = OUTLET;
    if (type == "symmetry") r.type = SYMMETRY;
    if (kind == "slip") r.kind = SLIP;
    r.area = 0.;
    r.total_area = 0.;
    for (int f = 0; f < g.faceCount; ++f) {
      if (g.face[f].bc == b) {
        g.face[f].symmetry = false;
        g.face2bc[f] = bc_counter[b];
        bc_counter[b]++;
        r.area += g.face[f].area;
        r.areaVec += g.face[f].area * g.face[f].normal;
        if (r.type == SYMMETRY) g.face[f].symmetry = true;
      }
    }
    r.total_area = r.area;
    O.bc.push_back(r);
  }
  g.boundaryFaceCount.assign(count, 0);
  for (int b = 0; b < count; ++b)
    for (int f = 0; f < g.faceCount; ++f)
      if (g.face[f].bc == b) g.boundaryFaceCount[b]++;
  int nsf = 0;
  for (int f = 0; f < g.faceCount; ++f) {
    if (g.face[f].bc == UNASSIGNED_FACE) throw DeckError("boundary condition could not be found for face " + std::to_string(f));
    if (g.face[f].bc >= 0) {
      const BCregion &r = O.bc[g.face[f].bc];
      if (r.type == WALL && r.kind != SLIP) nsf++;
      if (r.type == INLET || r.type == OUTLET) {
        int nb = g.face[f].neighbor, pa = g.face[f].parent;
        g.cell[nb].centroid = g.cell[pa].centroid + 2. * (g.face[f].centroid - g.cell[pa].centroid);
      }
    }
  }
  std::vector<double> wx, wy, wz, wnx, wny, wnz;
  for (int f = 0; f < g.faceCount; ++f) {
    if (g.face[f].bc >= 0 && O.bc[g.face[f].bc].type == WALL && O.bc[g.face[f].bc].kind != SLIP) {
      wx.push_back(g.face[f].centroid[0]); wy.push_back(g.face[f].centroid[1]); wz.push_back(g.face[f].centroid[2]);
      wnx.push_back(g.face[f].normal[0]); wny.push_back(g.face[f].normal[1]); wnz.push_back(g.face[f].normal[2]);
    }
  }
  (void)nsf;
  for (size_t c = 0; c < g.cell.size(); ++c) {
    g.cell[c].closest_wall_distance = 1.e20;
    for (size_t k = 0; k < wx.size(); ++k) {
      Vec3 t(wx[k], wy[k], wz[k]);
      double d = fabs(g.cell[c].centroid - t);
      if (g.cell[c].closest_wall_distance > d) g.cell[c].closest_wall_distance = d;
    }
  }
  for (int f = 0; f < g.faceCount; ++f) {
    Face &F = g.face[f];
    F.closest_wall_distance = 1.e20;
    if (F.bc < 0 || O.bc[F.bc].type != WALL || O.bc[F.bc].kind == SLIP) {
      Vec3 fN;
      for (size_t k = 0; k < wx.size(); ++k) {
        Vec3 t(wx[k], wy[k], wz[k]);
        double d = fabs(F.centroid - t);
        if (F.closest_wall_distance > d) { F.closest_wall_distance = d; fN = Vec3(wnx[k], wny[k], wnz[k]); }
      }
      F.dissipation_factor = 1. - std::fabs(fN[0] * F.normal[0] + fN[1] * F.normal[1] + fN[2] * F.normal[2]);
    } else {
      F.closest_wall_distance = 0.;
      F.dissipation_factor = 0.;
    }
  }
}

// main.cc:456-491
static void set_lengthScales(Oracle &O) {
  Grid &g = O.grid;
  for (int c = 0; c < g.cellCount; ++c) {
    g.cell[c].lengthScale = 1.e20;
    for (size_t cf = 0; cf < g.cell[c].faces.size(); ++cf) {
      int f = g.cell[c].faces[cf];
      double height = std::fabs(g.face[f].normal.dot(g.face[f].centroid - g.cell[c].centroid));
      bool skip = false;
      if (g.face[f].bc >= 0 && O.bc[g.face[f].bc].type == SYMMETRY) skip = true;
      if (!skip) g.cell[c].lengthScale = std::min(g.cell[c].lengthScale, height);
    }
  }
  if (g.dimension == 3) {
    g.lengthScale = std::pow(g.globalTotalVolume, 1. / 3.);
  } else {
    g.lengthScale = 0.;
    for (size_t b = 0; b < O.bc.size(); ++b)
      if (O.bc[b].type == SYMMETRY) g.lengthScale = std::max(g.lengthScale, std::sqrt(0.5 * O.bc[b].total_area));
  }
}

// face_interpolation_weights.cc:32-138 with interpolate.cc:36-119 (sort_stencil)
// and interpolate.cc:320-352 (line / point).  Triangle and tetrahedron
// interpolation (stencil size > 2) are not restated: decks must keep the
// default stencil size of 2 for WTLI.
static void face_interpolation_weights(Oracle &O) {
  Grid &g = O.grid;
  int max_stencil = O.stencil_size;
  if (max_stencil < 1) max_stencil = (g.dimension == 3) ? 12 : (g.dimension == 2 ? 6 : 2);
  if (O.interp_method == IDW) max_stencil = 99;
  for (int f = 0; f < g.faceCount; ++f) {
    Face &F = g.face[f];
    int c = F.parent, n = F.neighbor;
    std::vector<Vec3> stencil{g.cell[c].centroid, g.cell[n].centroid};
    std::vector<int> idx{c, n};
    bool extend = !((int)stencil.size() >= max_stencil);
    if (extend) {
      std::set<int> st;
      for (int k : g.cell[c].neighborCells) st.insert(k);
      if (F.bc == INTERNAL_FACE)
        for (int k : g.cell[F.neighbor].neighborCells) st.insert(k);
      st.erase(F.parent);
      st.erase(F.neighbor);
      for (int k : st) { idx.push_back(k); stencil.push_back(g.cell[k].centroid); }
    }
    if (O.interp_method == WTLI) {
      if (max_stencil > 2) throw DeckError("interpolation stencil size > 2 (tri/tetra WTLI) is not supported");
      // sort_stencil with is_internal=true keeps [parent, neighbor]; interpolate_line:
      Vec3 edge1 = stencil[1] - stencil[0];
      Vec3 basis1 = edge1;
      basis1 = basis1.norm();
      Vec3 p_point = F.centroid - stencil[0];
      p_point = p_point.dot(basis1) * basis1;
      double w1 = p_point.dot(basis1) / fabs(edge1);
      double w0 = 1. - w1;
      // weights are normalised by their sum only in the tri/tetra paths
      F.average.insert({idx[0], w0});
      F.average.insert({idx[1], w1});
    } else if (O.interp_method == IDW) {
      std::vector<double> w(stencil.size(), 0.);
      double sum = 0.;
      for (size_t s = 0; s < stencil.size(); ++s) { w[s] = fabs(F.centroid - stencil[s]); sum += w[s]; }
      for (size_t s = 0; s < stencil.size(); ++s) w[s] /= sum;
      for (size_t s = 0; s < stencil.size(); ++s) F.average.insert({idx[s], w[s]});
    } else {
      F.average.insert({idx[0], 0.5});
      F.average.insert({idx[1], 0.5});
    }
  }
}

// lsqr_grad_map.cc:32-99
static void lsqr_grad_map(Grid &g, int ci) {
  std::vector<int> stencil;
  std::vector<double> w;
  std::vector<Vec3> distance;
  for (int nb : g.cell[ci].neighborCells)
    if (nb != ci) stencil.push_back(nb);
  double a = 0., b = 0., c = 0., d = 0., e = 0, f = 0.;
  for (size_t k = 0; k < stencil.size(); k++) {
    Vec3 point = g.cell[stencil[k]].centroid;
    distance.push_back(point - g.cell[ci].centroid);
    w.push_back(distance[k].dot(distance[k]));
    a += w[k] * distance[k][0] * distance[k][0];
    b += w[k] * distance[k][0] * distance[k][1];
    c += w[k] * distance[k][0] * distance[k][2];
    d += w[k] * distance[k][1] * distance[k][1];
    e += w[k] * distance[k][1] * distance[k][2];
    f += w[k] * distance[k][2] * distance[k][2];
  }
  for (size_t cf = 0; cf < g.cell[ci].faces.size(); ++cf) {
    if (g.face[g.cell[ci].faces[cf]].symmetry) {
      stencil.push_back(ci);
      Vec3 point = g.cell[ci].centroid + (g.cellFace(ci, (int)cf).centroid - g.cell[ci].centroid).dot(g.cellFace(ci, (int)cf).normal) * g.cellFace(ci, (int)cf).normal;
      distance.push_back(point - g.cell[ci].centroid);
      size_t k = distance.size() - 1;
      w.push_back(distance[k].dot(distance[k]));
      a += w[k] * distance[k][0] * distance[k][0];
      b += w[k] * distance[k][0] * distance[k][1];
      c += w[k] * distance[k][0] * distance[k][2];
      d += w[k] * distance[k][1] * distance[k][1];
      e += w[k] * distance[k][1] * distance[k][2];
      f += w[k] * distance[k][2] * distance[k][2];
    }
  }
  double det = a * d * f - a * e * e - b * b * f - c * c * d + 2. * b * c * e;
  Vec3 weight;
  g.cell[ci].gradMap.clear();
  for (size_t k = 0; k < stencil.size(); k++) {
    weight[0] = w[k] * (distance[k][0] * (d * f - e * e) + distance[k][1] * (c * e - b * f) + distance[k][2] * (b * e - c * d));
    weight[1] = w[k] * (distance[k][0] * (c * e - b * f) + distance[k][1] * (a * f - c * c) + distance[k][2] * (b * c - a * e));
    weight[2] = w[k] * (distance[k][0] * (b * e - c * d) + distance[k][1] * (b * c - a * e) + distance[k][2] * (a * d - b * b));
    weight /= det;
    g.cell[ci].gradMap.insert({stencil[k], weight});
    if (g.cell[ci].gradMap.find(ci) == g.cell[ci].gradMap.end()) g.cell[ci].gradMap.insert({ci, -1. * weight});
    else g.cell[ci].gradMap[ci] -= weight;
  }
}

// curvilinear_grad_map.cc:28-228.  The hexahedron branch (lines 58-77)
// erases the std::set element its loop iterator points at and then
// increments that iterator (undefined behaviour); restated here is the
// pairing the loop is written to produce: the faces still unpaired, in
// ascending order, each paired with the later unpaired face whose outward
// normal is most opposite (first minimum).
static void curvilinear_grad_map(Grid &g, int c) {
  std::set<int> stencil;
  std::vector<int> face_pairs(6, -1), cell_pairs(6, -1), cell_pairs_temp(6, -1);
  std::vector<Vec3> Jac(3), Jac_temp(3), Jac_invT(3);
  double det;
  int cell_plus, cell_minus;
  for (int cf = 0; cf < (int)g.cell[c].faces.size(); ++cf) stencil.insert(cf);
  if (g.cell[c].nodes.size() == 8) {
    int counter = 0;
    while (!stencil.empty()) {
      std::set<int>::iterator sit1 = stencil.begin(), sit2;
      double min_product = 1.e20;
      Vec3 my_normal = g.cellFace(c, *sit1).normal;
      if (g.cellFace(c, *sit1).parent != c) my_normal *= -1.;
      face_pairs[2 * counter + 1] = *sit1;
      sit2 = sit1;
      sit2++;
      for (; sit2 != stencil.end(); sit2++) {
        Vec3 other_normal = g.cellFace(c, *sit2).normal;
        if (g.cellFace(c, *sit2).parent != c) other_normal *= -1.;
        double product = my_normal.dot(other_normal);
        if (product < min_product) {
          min_product = product;
          face_pairs[2 * counter] = *sit2;
        }
      }
      stencil.erase(face_pairs[2 * counter]);
      stencil.erase(face_pairs[2 * counter + 1]);
      counter++;
      if (counter == 3) break;
    }
    for (int i = 0; i < 3; ++i) {
      cell_plus = g.cellFace(c, face_pairs[2 * i + 1]).neighbor;
      if (cell_plus == c) cell_plus = g.cellFace(c, face_pairs[2 * i + 1]).parent;
      cell_pairs[2 * i + 1] = cell_plus;
      Jac[i] = g.cell[cell_plus].centroid;
      cell_minus = g.cellFace(c, face_pairs[2 * i]).neighbor;
      if (cell_minus == c) cell_minus = g.cellFace(c, face_pairs[2 * i]).parent;
      cell_pairs[2 * i] = cell_minus;
      Jac[i] -= g.cell[cell_minus].centroid;
    }
  } else {
    double max_det = 0.;
    stencil.clear();
    for (int cf = 0; cf < (int)g.cell[c].faces.size(); ++cf) stencil.insert(g.cell[c].faces[cf]);
    std::set<int>::iterator sit1, sit2, sit3, sit4, sit5, sit6;
    for (sit1 = stencil.begin(); sit1 != stencil.end(); sit1++) {
      for (sit2 = sit1; sit2 != stencil.end(); sit2++) {
        cell_plus = g.face[*sit2].neighbor;
        if (cell_plus == c) cell_plus = g.face[*sit2].parent;
        cell_pairs_temp[1] = cell_plus;
        Jac_temp[0] = g.cell[cell_plus].centroid;
        cell_minus = g.face[*sit1].neighbor;
        if (cell_minus == c) cell_minus = g.face[*sit1].parent;
        cell_pairs_temp[0] = cell_minus;
        Jac_temp[0] -= g.cell[cell_minus].centroid;
        for (sit3 = sit1; sit3 != stencil.end(); sit3++) {
          for (sit4 = sit3; sit4 != stencil.end(); sit4++) {
            cell_plus = g.face[*sit4].neighbor;
            if (cell_plus == c) cell_plus = g.face[*sit4].parent;
            cell_pairs_temp[3] = cell_plus;
            Jac_temp[1] = g.cell[cell_plus].centroid;
            cell_minus = g.face[*sit3].neighbor;
            if (cell_minus == c) cell_minus = g.face[*sit3].parent;
            cell_pairs_temp[2] = cell_minus;
            Jac_temp[1] -= g.cell[cell_minus].centroid;
            for (sit5 = sit2; sit5 != stencil.end(); sit5++) {
              for (sit6 = sit5; sit6 != stencil.end(); sit6++) {
                cell_plus = g.face[*sit6].neighbor;
                if (cell_plus == c) cell_plus = g.face[*sit6].parent;
                cell_pairs_temp[5] = cell_plus;
                Jac_temp[2] = g.cell[cell_plus].centroid;
                cell_minus = g.face[*sit5].neighbor;
                if (cell_minus == c) cell_minus = g.face[*sit5].parent;
                cell_pairs_temp[4] = cell_minus;
                Jac_temp[2] -= g.cell[cell_minus].centroid;
                det = Jac_temp[0].dot(Jac_temp[1].cross(Jac_temp[2]));
                if (det > max_det) {
                  max_det = det;
                  cell_pairs = cell_pairs_temp;
                  Jac = Jac_temp;
                }
              }
            }
          }
        }
      }
    }
    if (!(max_det > 0.)) throw DeckError("curvilinear gradient: no face pairs with a positive determinant");
  }
  det = Jac[0].dot(Jac[1].cross(Jac[2]));
  Jac_invT[0][0] = (Jac[1][1] * Jac[2][2] - Jac[1][2] * Jac[2][1]) / det;
  Jac_invT[1][0] = (Jac[0][2] * Jac[2][1] - Jac[0][1] * Jac[2][2]) / det;
  Jac_invT[2][0] = (Jac[0][1] * Jac[1][2] - Jac[0][2] * Jac[1][1]) / det;
  Jac_invT[0][1] = (Jac[1][2] * Jac[2][0] - Jac[1][0] * Jac[2][2]) / det;
  Jac_invT[1][1] = (Jac[0][0] * Jac[2][2] - Jac[0][2] * Jac[2][0]) / det;
  Jac_invT[2][1] = (Jac[0][2] * Jac[1][0] - Jac[0][0] * Jac[1][2]) / det;
  Jac_invT[0][2] = (Jac[1][0] * Jac[2][1] - Jac[1][1] * Jac[2][0]) / det;
  Jac_invT[1][2] = (Jac[0][1] * Jac[2][0] - Jac[0][0] * Jac[2][1]) / det;
  Jac_invT[2][2] = (Jac[0][0] * Jac[1][1] - Jac[0][1] * Jac[1][0]) / det;
  std::map<int, Vec3> gradMap;
  gradMap.insert(std::pair<int, Vec3>(cell_pairs[0], -1. * Jac_invT[0]));
  if (gradMap.find(cell_pairs[1]) == gradMap.end()) gradMap.insert(std::pair<int, Vec3>(cell_pairs[1], Jac_invT[0]));
  else gradMap[cell_pairs[1]] += Jac_invT[0];
  if (gradMap.find(cell_pairs[2]) == gradMap.end()) gradMap.insert(std::pair<int, Vec3>(cell_pairs[2], -1. * Jac_invT[1]));
  else gradMap[cell_pairs[2]] -= Jac_invT[1];
  if (gradMap.find(cell_pairs[3]) == gradMap.end()) gradMap.insert(std::pair<int, Vec3>(cell_pairs[3], Jac_invT[1]));
  else gradMap[cell_pairs[3]] += Jac_invT[1];
  if (gradMap.find(cell_pairs[4]) == gradMap.end()) gradMap.insert(std::pair<int, Vec3>(cell_pairs[4], -1. * Jac_invT[2]));
  else gradMap[cell_pairs[4]] -= Jac_invT[2];
  if (gradMap.find(cell_pairs[5]) == gradMap.end()) gradMap.insert(std::pair<int, Vec3>(cell_pairs[5], Jac_invT[2]));
  else gradMap[cell_pairs[5]] += Jac_invT[2];
  g.cell[c].gradMap = gradMap;
}

// gradient_maps.cc:39-78
static void gradient_maps(Oracle &O) {
  Grid &g = O.grid;
  for (int c = 0; c < g.cellCount; ++c) {
    int m = (g.cell[c].nodes.size() == 8) ? O.hex_method : (g.cell[c].nodes.size() == 6 ? O.prism_method : O.other_method);
    if (m == CURVILINEAR) curvilinear_grad_map(g, c);
    if (m == LSQR) lsqr_grad_map(g, c);
  }
}

static int method_of(const std::string &s) {
  if (s == "curvilinear") return CURVILINEAR;
  if (s == "lsqr") return LSQR;
  if (s == "greengauss") return GREENGAUSS;
  return CURVILINEAR;
}

// ns.cc:33-102 options, material.cc:29-106, ns_set_bcs.cc:25-140
static void setup_physics(Oracle &O, const std::string &deck_dir) {
  Section &g = O.input.section("grid", 0);
  Subsection &ns = g.sub("navierstokes");
  std::string lim = ns.gs("limiter").value;
  O.limiter_function = (lim == "vk") ? VK : (lim == "bj") ? BJ : (lim == "minmod") ? MINMOD : NONE;
  O.limiter_threshold = ns.gd("limiterthreshold").value;
  std::string ord = ns.gs("order").value;
  if (ord == "first") O.order = FIRST;
  else if (ord == "second") O.order = SECOND;
  std::string fl = ns.gs("convectiveflux").value;
  if (fl == "AUSM+up") O.flux = AUSM_PLUS_UP;
  else if (fl == "Roe") O.flux = ROE;
  else if (fl == "vanLeer") O.flux = VAN_LEER;
  else if (fl == "SD-SLAU") O.flux = SD_SLAU;
  else if (fl == "SW") O.flux = SW;
  else throw DeckError("convective flux " + fl + " is not on the restated path");
  O.Minf = O.input.section("reference").gd("Mach").value;
  {
    const V3d &mc = g.sub("writeoutput").gv("momentcenter").value;
    O.moment_center = Vec3(mc.c[0], mc.c[1], mc.c[2]);
  }
  O.wdiss = ns.gd("walldissipation").value;
  O.bl_height = ns.gd("BLheight").value;
  O.hex_method = method_of(g.sub("gradients").gs("hexmethod").value);
  O.prism_method = method_of(g.sub("gradients").gs("prismmethod").value);
  O.other_method = method_of(g.sub("gradients").gs("othermethod").value);
  std::string im = g.sub("interpolation").gs("method").value;
  O.interp_method = (im == "idw") ? IDW : (im == "simple") ? SIMPLE : WTLI;
  O.stencil_size = g.sub("interpolation").gi("stencilsize").value;
  O.grid.dimension = g.gi("dimension").value;

  Material &m = O.material;
  if (g.gs("material").is_found) {
    std::string fn = g.gs("material").value + ".mat";
    std::string path = deck_dir.empty() ? fn : deck_dir + "/" + fn;
    O.matfile.setFile(path);
    register_material_schema(O.matfile);
    InputFile &mi = O.matfile;
    m.Mw = mi.gd("molarmass").value;
    m.gamma = mi.gd("gamma").value;
    if (mi.section("equationofstate").gs("model").value != "idealgas") throw DeckError("invalid equation of state option");
    m.R = 8314.47215 / m.Mw;
    if (mi.gd("viscosity").is_found) { m.sutherland = false; m.mu = mi.gd("viscosity").value; }
    else if (mi.section("viscosity").is_found) {
      if (mi.section("viscosity").gs("model").value != "sutherlands") throw DeckError("invalid viscosity model");
      m.sutherland = true;
      m.sut_mu_ref = mi.section("viscosity").gd("referenceviscosity").value;
      m.sut_T_ref = mi.section("viscosity").gd("referencetemperature").value;
      m.sut_S = mi.section("viscosity").gd("sutherlandtemperature").value;
    }
    if (mi.gd("thermalconductivity").is_found) { m.prandtl = false; m.lambda = mi.gd("thermalconductivity").value; }
    else if (mi.section("thermalconductivity").is_found) {
      if (mi.section("thermalconductivity").gs("model").value != "constantPrandtl") throw DeckError("invalid thermal conductivity model");
      m.prandtl = true;
      m.Pr = mi.section("thermalconductivity").gd("Pr").value;
    }
  } else {
    Subsection &ms = g.sub("material");
    m.Mw = ms.gd("molarmass").value;
    m.R = 8314.47215 / m.Mw;
    m.gamma = ms.gd("gamma").value;
    m.sutherland = false;
    m.mu = ms.gd("viscosity").value;
    m.prandtl = false;
    m.lambda = ms.gd("thermalconductivity").value;
  }
  m.Pref = O.input.section("reference").gd("p").value;
  m.Tref = O.input.section("reference").gd("T").value;

  // Time step options (time_step.cc:25-86)
  Section &tm = O.input.section("timemarching");
  O.has_cfl_max = tm.gd("CFLmax").is_found;
  O.has_cfl_local = tm.gd("CFLlocal").is_found;
  O.cfl_max = tm.gd("CFLmax").value;
  O.cfl_local = tm.gd("CFLlocal").value;

  // NavierStokes::set_bcs (ns_set_bcs.cc:25-140)
  int count = g.sub("BC", 0).count;
  O.p_fixed.assign(count, 0); O.T_fixed.assign(count, 0); O.rho_fixed.assign(count, 0); O.V_fixed.assign(count, 0);
  O.qdot_fixed.assign(count, 0); O.mdot_fixed.assign(count, 0); O.pt_fixed.assign(count, 0); O.Tt_fixed.assign(count, 0);
  O.p_bc.assign(count, 0.); O.T_bc.assign(count, 0.); O.rho_bc.assign(count, 0.); O.qdot_bc.assign(count, 0.);
  O.mdot_bc.assign(count, 0.); O.pt_bc.assign(count, 0.); O.Tt_bc.assign(count, 0.); O.V_bc.assign(count, Vec3());
  for (int b = 0; b < count; ++b) {
    Subsection &region = g.sub("BC", b);
    BCregion &r = O.bc[b];
    std::string kind = region.gs("kind").value;
    if (kind == "none") r.kind = NONE;
    if (kind == "noreverse") r.kind = NO_REVERSE;
    if (kind == "dampreverse") r.kind = DAMP_REVERSE;
    if (kind == "slip") r.kind = SLIP;
    if (kind == "forcesupersonic") r.kind = FORCE_SUPERSONIC;
    if (region.gd("p_total").is_found && region.gd("T_total").is_found) {
      r.kind = STAGNATION;
      O.pt_fixed[b] = 1; O.pt_bc[b] = region.gd("p_total").value;
      O.Tt_fixed[b] = 1; O.Tt_bc[b] = region.gd("T_total").value;
    }
    if (region.gd("p").is_found) {
      O.p_fixed[b] = 1; O.p_bc[b] = region.gd("p").value; r.specified = BC_P;
      if (region.gd("T").is_found) {
        if (region.gd("rho").is_found) throw DeckError("thermodynamic state is overspecified");
        O.T_fixed[b] = 1; O.T_bc[b] = region.gd("T").value;
        O.rho_fixed[b] = 1; O.rho_bc[b] = m.rho(O.p_bc[b], O.T_bc[b]);
        r.thermalType = FIXED_T; r.specified = BC_STATE;
      } else if (region.gd("rho").is_found) {
        O.rho_fixed[b] = 1; O.rho_bc[b] = region.gd("rho").value;
        O.T_fixed[b] = 1; O.T_bc[b] = m.temp(O.p_bc[b], O.rho_bc[b]);
        r.thermalType = FIXED_T; r.specified = BC_STATE;
      } else {
        if (r.type == WALL) r.thermalType = ADIABATIC;
      }
    } else if (region.gd("T").is_found) {
      O.T_fixed[b] = 1; O.T_bc[b] = region.gd("T").value;
      r.thermalType = FIXED_T; r.specified = BC_T;
      if (region.gd("rho").is_found) {
        O.rho_fixed[b] = 1; O.rho_bc[b] = region.gd("rho").value;
        O.p_fixed[b] = 1; O.p_bc[b] = m.pres(O.rho_bc[b], O.T_bc[b]);
        r.specified = BC_STATE;
      }
    } else if (region.gd("rho").is_found) {
      O.rho_fixed[b] = 1; O.rho_bc[b] = region.gd("rho").value;
      r.specified = BC_RHO;
    } else {
      if (r.type == WALL) r.thermalType = ADIABATIC;
    }
    if (region.gd("qdot").is_found) {
      if (r.type == WALL) {
        if (region.gd("T").is_found) throw DeckError("can't specify both temperature and qdot");
        r.thermalType = FIXED_Q;
        O.qdot_fixed[b] = 1; O.qdot_bc[b] = region.gd("qdot").value;
      }
    }
    if (r.type == WALL && r.kind != SLIP) { O.V_fixed[b] = 1; O.V_bc[b] = Vec3(0., 0., 0.); }
    if (r.type == SYMMETRY) r.thermalType = ADIABATIC;
    if (region.gv("V").is_found) {
      O.V_fixed[b] = 1;
      const V3d &v = region.gv("V").value;
      O.V_bc[b] = Vec3(v.c[0], v.c[1], v.c[2]);
      r.kind = VELOCITY;
    }
    if (region.gd("mdot").is_found) {
      r.kind = MDOT;
      O.mdot_fixed[b] = 1; O.mdot_bc[b] = region.gd("mdot").value;
    }
  }
}

// ================================================================ residual path (templated on S)

template <class S>
struct Fields {
  std::vector<S> p, T, rho;
  std::vector<V3<S>> V, gradp, gradu, gradv, gradw, gradT;
  std::vector<S> limiter[5];
  std::vector<S> mdot, weightL;
  S qmax[5], qmin[5];
  void alloc(size_t ncell, size_t nface) {
    p.assign(ncell, S(0.)); T.assign(ncell, S(0.)); rho.assign(ncell, S(0.));
    V.assign(ncell, V3<S>()); gradp.assign(ncell, V3<S>()); gradu.assign(ncell, V3<S>());
    gradv.assign(ncell, V3<S>()); gradw.assign(ncell, V3<S>()); gradT.assign(ncell, V3<S>());
    for (int i = 0; i < 5; ++i) limiter[i].assign(ncell, S(1.));
    mdot.assign(nface, S(0.)); weightL.assign(nface, S(0.));
  }
};

template <class S>
struct NS {
  Oracle &O;
  Fields<S> &F;
  CellState<S> left, right;  // the reference's namespace-scope state caches (ns_assemble_linear_system.cc:25-31)
  FaceState<S> face;
  NS(Oracle &o, Fields<S> &f) : O(o), F(f) {}

  // Variable<double>::cell_gradient (variable.h:193-216) for scalars
  // which: 0 p, 1 T (their BC-fixed face values), 2 neither
  V3<S> scalar_gradient(const std::vector<S> &phi, int c, int which = 2) {
    V3<S> grad;
    Grid &g = O.grid;
    if (!g.cell[c].gradMap.empty()) {
      for (auto &kv : g.cell[c].gradMap)
        for (int i = 0; i < 3; ++i) grad[i] += kv.second[i] * phi[kv.first];
    } else {
      for (size_t cf = 0; cf < g.cell[c].faces.size(); ++cf) {
        int f = g.cell[c].faces[cf];
        Vec3 areaVec = g.face[f].normal * g.face[f].area / g.cell[c].volume;
        if (g.face[f].parent != c) areaVec *= -1.;
        S fv = face_scalar(phi, f, which);
        for (int i = 0; i < 3; ++i) grad[i] += fv * areaVec[i];
      }
    }
    return grad;
  }
  // Variable<double>::face_calculate (variable.h:134-147); which: 0 p, 1 T
  S face_scalar(const std::vector<S> &phi, int f, int which) {
    Grid &g = O.grid;
    int b = g.face[f].bc;
    if (b >= 0) {
      if (which == 0 && O.p_fixed[b]) return S(O.p_bc[b]);
      if (which == 1 && O.T_fixed[b]) return S(O.T_bc[b]);
    }
    S t(0.);
    for (auto &kv : g.face[f].average) t += kv.second * phi[kv.first];
    return t;
  }
  // Variable<Vec3D>::face_calculate for a gradient variable (never fixed on a BC)
  V3<S> face_vec(const std::vector<V3<S>> &v, int f) {
    V3<S> t;
    for (auto &kv : O.grid.face[f].average) t = vadd(t, vscale(kv.second, v[kv.first]));
    return t;
  }

  // ns.cc:301-336
  void calc_cell_grads() {
    Grid &g = O.grid;
    for (int c = 0; c < g.cellCount; ++c) {
      F.gradp[c] = scalar_gradient(F.p, c, 0);
      F.gradT[c] = scalar_gradient(F.T, c, 1);
      V3<S> gx, gy, gz;  // V.cell_gradient(c): grad[i] is a Vec3D (d/dx_i of V)
      if (!g.cell[c].gradMap.empty()) {
        for (auto &kv : g.cell[c].gradMap) {
          gx = vadd(gx, vscale(kv.second[0], F.V[kv.first]));
          gy = vadd(gy, vscale(kv.second[1], F.V[kv.first]));
          gz = vadd(gz, vscale(kv.second[2], F.V[kv.first]));
        }
      } else {
        // Green-Gauss fallback (variable.h:204-213) for the Vec3D variable:
        // d/dx_i of V += V.face(f) * areaVec[i], V.face the BC value where V
        // is fixed on the BC, else the face average
        for (size_t cf = 0; cf < g.cell[c].faces.size(); ++cf) {
          int f = g.cell[c].faces[cf];
          Vec3 areaVec = g.face[f].normal * g.face[f].area / g.cell[c].volume;
          if (g.face[f].parent != c) areaVec *= -1.;
          const int b = g.face[f].bc;
          V3<S> Vf;
          if (b >= 0 && O.V_fixed[b]) Vf = V3<S>(S(O.V_bc[b][0]), S(O.V_bc[b][1]), S(O.V_bc[b][2]));
          else Vf = face_vec(F.V, f);
          gx = vadd(gx, vscale(areaVec[0], Vf));
          gy = vadd(gy, vscale(areaVec[1], Vf));
          gz = vadd(gz, vscale(areaVec[2], Vf));
        }
      }
      F.gradu[c] = V3<S>(gx[0], gy[0], gz[0]);
      F.gradv[c] = V3<S>(gx[1], gy[1], gz[1]);
      F.gradw[c] = V3<S>(gx[2], gy[2], gz[2]);
    }
    for (int f = 0; f < g.faceCount; ++f) {
      if (g.face[f].bc >= 0) {
        int pa = g.face[f].parent, nb = g.face[f].neighbor;
        F.gradp[nb] = F.gradp[pa]; F.gradu[nb] = F.gradu[pa]; F.gradv[nb] = F.gradv[pa];
        F.gradw[nb] = F.gradw[pa]; F.gradT[nb] = F.gradT[pa];
      }
    }
  }

  // ns.cc:400-435 (index quirks kept: qmax[3] reads qmax[4]; index 4 tracks p)
  void find_min_max() {
    F.qmax[0] = F.qmin[0] = F.p[0];
    F.qmax[1] = F.qmin[1] = F.V[0][0];
    F.qmax[2] = F.qmin[2] = F.V[0][1];
    F.qmax[3] = F.qmin[3] = F.V[0][2];
    F.qmax[4] = F.qmin[4] = F.T[0];
    for (int c = 0; c < O.grid.cellCount; ++c) {
      F.qmax[0] = smax(F.qmax[0], F.p[c]);
      F.qmax[1] = smax(F.qmax[1], F.V[c][0]);
      F.qmax[2] = smax(F.qmax[2], F.V[c][1]);
      F.qmax[3] = smax(F.qmax[4], F.V[c][2]);
      F.qmax[4] = smax(F.qmax[4], F.p[c]);
      F.qmin[0] = smin(F.qmin[0], F.p[c]);
      F.qmin[1] = smin(F.qmin[1], F.V[c][0]);
      F.qmin[2] = smin(F.qmin[2], F.V[c][1]);
      F.qmin[3] = smin(F.qmin[4], F.V[c][2]);
      F.qmin[4] = smin(F.qmin[4], F.p[c]);
    }
  }

  S var_of(int var, int c) {
    switch (var) {
      case 0: return F.p[c];
      case 1: return F.V[c][0];
      case 2: return F.V[c][1];
      case 3: return F.V[c][2];
      default: return F.T[c];
    }
  }
  const V3<S> &grad_of(int var, int c) {
    switch (var) {
      case 0: return F.gradp[c];
      case 1: return F.gradu[c];
      case 2: return F.gradv[c];
      case 3: return F.gradw[c];
      default: return F.gradT[c];
    }
  }

  // ns_limiters.cc:161-248
  void venkatakrishnan_limiter() {
    Grid &g = O.grid;
    find_min_max();
    double K = O.limiter_threshold;
    double Lref = g.lengthScale;
    S deltaRef[5];
    for (int i = 0; i < 5; ++i) deltaRef[i] = fabs(F.qmax[i] - F.qmin[i]);
    for (int c = 0; c < g.cellCount; ++c) {
      S phi[5], umax[5], umin[5];
      for (int i = 0; i < 5; ++i) { phi[i] = S(1.); umax[i] = umin[i] = var_of(i, c); }
      for (size_t cf = 0; cf < g.cell[c].faces.size(); ++cf) {
        const Face &Fc = g.cellFace(c, (int)cf);
        int nb = (c == Fc.parent) ? Fc.neighbor : Fc.parent;
        for (int i = 0; i < 5; ++i) { umax[i] = smax(umax[i], var_of(i, nb)); umin[i] = smin(umin[i], var_of(i, nb)); }
      }
      for (size_t cf = 0; cf < g.cell[c].faces.size(); ++cf) {
        Vec3 cell2face = g.cellFace(c, (int)cf).centroid - g.cell[c].centroid;
        for (int var = 0; var < 5; ++var) {
          S deltaM = vdot(grad_of(var, c), cell2face);
          S deltaP = var_of(var, c);
          S eps = deltaRef[var] / Lref;
          if (deltaM > 0.) deltaP = umax[var] - deltaP;
          else if (deltaM < 0.) deltaP = umin[var] - deltaP;
          S deltaP2 = deltaP * deltaP;
          S deltaM2 = deltaM * deltaM;
          S e = 1.e-6 * K * eps;
          S eps2 = e * e;  // pow(x,2)
          if (deltaM != 0.)
            phi[var] = smin(phi[var], ((deltaP2 + eps2) + 2. * deltaM * deltaP) / (deltaP2 + 2. * deltaM2 + deltaM * deltaP + eps2));
        }
      }
      for (int var = 0; var < 5; ++var) F.limiter[var][c] = phi[var];
    }
  }

  static S minmod(const S &a1, const S &a2) {  // ns_limiters.cc:39-43
    if (a1 * a2 < 0.) return S(0.);
    else if (a1 > 0.) return smin(a1, a2);
    else return smax(a1, a2);
  }
  static double sgn(const S &x) { double r = re_(x); return double((r > 0) - (r < 0)); }

  // ns_limiters.cc:45-92
  void minmod_limiter() {
    Grid &g = O.grid;
    const double small = 1.e-12;
    for (int c = 0; c < g.cellCount; ++c) {
      S phi[5];
      for (int i = 0; i < 5; ++i) phi[i] = S(1.);
      for (size_t cf = 0; cf < g.cell[c].faces.size(); ++cf) {
        const Face &Fc = g.cellFace(c, (int)cf);
        Vec3 cell2face = Fc.centroid - g.cell[c].centroid;
        int nb = (c == Fc.parent) ? Fc.neighbor : Fc.parent;
        for (int var = 0; var < 5; ++var) {
          S dU = var_of(var, nb) - var_of(var, c);
          S dUg = vdot(grad_of(var, c), cell2face);
          dU = minmod(dU, dUg);
          phi[var] = smin(phi[var], (dU + sgn(dU) * small) / (dUg + sgn(dUg) * small));
        }
      }
      for (int var = 0; var < 5; ++var) F.limiter[var][c] = phi[var];
    }
  }

  // ns_limiters.cc:94-159
  void barth_jespersen_limiter() {
    Grid &g = O.grid;
    for (int c = 0; c < g.cellCount; ++c) {
      S phi[5], umax[5], umin[5];
      for (int i = 0; i < 5; ++i) { phi[i] = S(1.); umax[i] = umin[i] = var_of(i, c); }
      for (size_t cf = 0; cf < g.cell[c].faces.size(); ++cf) {
        const Face &Fc = g.cellFace(c, (int)cf);
        int nb = (c == Fc.parent) ? Fc.neighbor : Fc.parent;
        for (int i = 0; i < 5; ++i) { umax[i] = smax(umax[i], var_of(i, nb)); umin[i] = smin(umin[i], var_of(i, nb)); }
      }
      for (size_t cf = 0; cf < g.cell[c].faces.size(); ++cf) {
        Vec3 cell2face = g.cellFace(c, (int)cf).centroid - g.cell[c].centroid;
        for (int var = 0; var < 5; ++var) {
          S deltaM = vdot(grad_of(var, c), cell2face);
          S deltaP = var_of(var, c);
          if (deltaM > 0.) deltaP = umax[var] - deltaP;
          else if (deltaM < 0.) deltaP = umin[var] - deltaP;
          else { deltaP = S(1.); deltaM = S(1.); }
          phi[var] = smin(phi[var], deltaP / deltaM);
        }
      }
      for (int var = 0; var < 5; ++var) F.limiter[var][c] = phi[var];
    }
  }

  void calc_limiter() {  // ns_limiters.cc:26-37
    if (O.limiter_function == NONE || O.order == FIRST) return;
    if (O.limiter_function == VK) venkatakrishnan_limiter();
    else if (O.limiter_function == BJ) barth_jespersen_limiter();
    else if (O.limiter_function == MINMOD) minmod_limiter();
  }

  // ns_assemble_linear_system.cc:332-351
  void face_geom_update(int f) {
    Grid &g = O.grid;
    face.index = f;
    face.parent = g.face[f].parent;
    face.neighbor = g.face[f].neighbor;
    face.normal = g.face[f].normal;
    if (g.face[f].nodes.size() == 4)
      face.tangent1 = ((Vec3(g.faceNode(f, 0)) + Vec3(g.faceNode(f, 1))) - (Vec3(g.faceNode(f, 2)) + Vec3(g.faceNode(f, 3)))).norm();
    else
      face.tangent1 = (0.5 * (Vec3(g.faceNode(f, 0)) + Vec3(g.faceNode(f, 1))) - g.face[f].centroid).norm();
    face.tangent2 = ((face.normal).cross(face.tangent1)).norm();
    face.area = g.face[f].area;
    face.bc = g.face[f].bc;
    face.left2right = g.cell[face.neighbor].centroid - g.cell[face.parent].centroid;
  }

  void finish_state(CellState<S> &st) {
    st.a = O.material.a(st.p, st.T);
    st.H = st.a * st.a / (O.material.gamma - 1.) + 0.5 * vdot(st.V, st.V);
    st.Vn[0] = vdot(st.V, face.normal);
    st.Vn[1] = vdot(st.V, face.tangent1);
    st.Vn[2] = vdot(st.V, face.tangent2);
  }

  // ns_assemble_linear_system.cc:269-294
  void left_state_update(CellState<S> &L) {
    Grid &g = O.grid;
    int pa = face.parent;
    Vec3 cell2face = 1. * g.face[face.index].centroid - g.cell[pa].centroid;  // order_factor=1
    L.p_center = F.p[pa];
    L.p = L.p_center + F.limiter[0][pa] * vdot(cell2face, F.gradp[pa]);
    V3<S> dV(F.limiter[1][pa] * vdot(cell2face, F.gradu[pa]), F.limiter[2][pa] * vdot(cell2face, F.gradv[pa]),
             F.limiter[3][pa] * vdot(cell2face, F.gradw[pa]));
    L.V_center = F.V[pa];
    L.V = vadd(L.V_center, dV);
    L.T_center = F.T[pa];
    L.T = L.T_center + F.limiter[4][pa] * vdot(cell2face, F.gradT[pa]);
    L.rho = O.material.rho(L.p, L.T);
    L.volume = g.cell[pa].volume;
    finish_state(L);
  }

  // ns_assemble_linear_system.cc:296-330
  void right_state_update(CellState<S> &L, CellState<S> &R) {
    Grid &g = O.grid;
    if (face.bc >= 0) {
      R.p_center = F.p[face.neighbor];
      R.T_center = F.T[face.neighbor];
      R.V_center = F.V[face.neighbor];
      apply_bcs(L, R);
    } else {
      int nb = face.neighbor;
      Vec3 cell2face = 1. * g.face[face.index].centroid - g.cell[nb].centroid;
      R.p_center = F.p[nb];
      R.p = R.p_center + F.limiter[0][nb] * vdot(cell2face, F.gradp[nb]);
      V3<S> dV(F.limiter[1][nb] * vdot(cell2face, F.gradu[nb]), F.limiter[2][nb] * vdot(cell2face, F.gradv[nb]),
               F.limiter[3][nb] * vdot(cell2face, F.gradw[nb]));
      R.V_center = F.V[nb];
      R.V = vadd(R.V_center, dV);
      R.T_center = F.T[nb];
      R.T = R.T_center + F.limiter[4][nb] * vdot(cell2face, F.gradT[nb]);
      R.rho = O.material.rho(R.p, R.T);
      R.volume = g.cell[nb].volume;
    }
    finish_state(R);
  }

  // ns_apply_bcs.cc:25-258
  void apply_bcs(CellState<S> &L, CellState<S> &R) {
    const BCregion &r = O.bc[face.bc];
    bool is_slip = (r.kind == SLIP);
    if (r.type == INLET) {
      if (r.kind == VELOCITY) velocity_inlet(L, R);
      else if (r.kind == MDOT) mdot_inlet(L, R);
      else if (r.kind == STAGNATION) stagnation_inlet(L, R);
    } else if (r.type == OUTLET) {
      outlet(L, R);
    } else if (r.type == WALL) {
      wall(L, R, is_slip);
    } else if (r.type == SYMMETRY) {
      symmetry(L, R);
    }
  }
  void velocity_inlet(CellState<S> &L, CellState<S> &R) {
    const Material &m = O.material;
    int b = face.bc;
    R.V = V3<S>(O.V_bc[b]);
    S uNL = vdot(L.V, face.normal);
    S uNR = vdot(R.V, face.normal);
    R.a = L.a + 0.5 * (uNL - uNR) * (m.gamma - 1.);
    S MachL = -uNL / L.a;
    if (MachL >= 1. && O.bc[b].specified != BC_STATE) throw DeckError("inlet became supersonic, need to specify the thermodynamic state");
    int sp = O.bc[b].specified;
    if (sp == BC_STATE) { R.p = S(O.p_bc[b]); R.T = S(O.T_bc[b]); R.rho = S(O.rho_bc[b]); }
    else if (sp == BC_P) { R.p = S(O.p_bc[b]); R.rho = m.gamma * (R.p + m.Pref) / (R.a * R.a); R.T = m.temp(R.p, R.rho); }
    else if (sp == BC_T) {
      R.T = S(O.T_bc[b]);
      R.rho = L.rho * pow((L.T + m.Tref) / (R.T + m.Tref), 1. / (1. - m.gamma));
      R.p = m.pres(R.rho, R.T);
    } else if (sp == BC_RHO) { R.rho = S(O.rho_bc[b]); R.p = R.a * R.a * R.rho / m.gamma - m.Pref; R.T = m.temp(R.p, R.rho); }
    else throw DeckError("at least one of p,T,rho needs to be specified at inlet");
    R.p_center = R.p; R.V_center = R.V; R.T_center = R.T;
  }
  void mdot_inlet(CellState<S> &L, CellState<S> &R) {
    const Material &m = O.material;
    int b = face.bc;
    S uNL = vdot(L.V, face.normal);
    double mdotNR = -1. * O.mdot_bc[b] / O.bc[b].total_area;
    int sp = O.bc[b].specified;
    if (sp == BC_STATE) { R.p = S(O.p_bc[b]); R.T = S(O.T_bc[b]); R.rho = S(O.rho_bc[b]); }
    else if (sp == BC_P) { R.p = S(O.p_bc[b]); R.T = L.T; R.rho = m.rho(R.p, R.T); }
    else if (sp == BC_T) { R.T = S(O.T_bc[b]); R.p = L.p; R.rho = m.rho(R.p, R.T); }
    else if (sp == BC_RHO) {
      R.rho = S(O.rho_bc[b]);
      R.a = 0.5 * (m.gamma - 1.) * (uNL + 2. * L.a / (m.gamma - 1.) - mdotNR / R.rho);
      R.p = R.a * R.a * R.rho / m.gamma - m.Pref;
      R.T = m.temp(R.p, R.rho);
    } else throw DeckError("at least one of p,T,rho needs to be specified at inlet");
    R.V = vscale(mdotNR / R.rho, face.normal);
    R.p_center = R.p; R.V_center = R.V; R.T_center = R.T;
  }
  void stagnation_inlet(CellState<S> &L, CellState<S> &R) {
    const Material &m = O.material;
    int b = face.bc;
    if (vdot(L.V, face.normal) > 0.) R.V = vscale(-1., L.V_center);
    else R.V = L.V_center;
    R.T = O.Tt_bc[b] - 0.5 * (m.gamma - 1.) / (m.gamma * m.R) * vdot(R.V, R.V);
    R.p = (O.pt_bc[b] + m.Pref) / (1. + 0.5 * vdot(R.V, R.V) / (m.R * (R.T + m.Tref))) - m.Pref;
    R.rho = m.rho(R.p, R.T);
    R.p_center = R.p; R.V_center = R.V; R.T_center = R.T;
  }
  void outlet(CellState<S> &L, CellState<S> &R) {
    const Material &m = O.material;
    int b = face.bc;
    const BCregion &r = O.bc[b];
    S uNL = vdot(L.V, face.normal);
    S MachL = uNL / L.a;
    bool supersonic = (MachL > 1.);
    if (r.specified == BC_STATE) throw DeckError("can't specify complete thermodynamic state at outlet");
    else if (r.specified == BC_P && !supersonic) {
      R.p = R.p_center = S(O.p_bc[b]);
      R.rho = L.rho * pow((R.p + m.Pref), 1. / m.gamma) / pow((L.p + m.Pref), 1. / m.gamma);
      R.a = sqrt(m.gamma * (R.p + m.Pref) / R.rho);
      R.T = m.temp(R.p, R.rho);
      R.V = L.V;
    } else if (r.specified == BC_T && !supersonic) {
      R.T = R.T_center = S(O.T_bc[b]);
      R.a = sqrt(m.gamma * m.R * (R.T + m.Tref));
      R.rho = pow(m.gamma * (L.p + m.Pref) / (R.a * R.a * pow(L.rho, m.gamma)), 1. - m.gamma);
      R.p = m.pres(R.rho, R.T);
      R.V = L.V;
    } else if (r.specified == BC_RHO && !supersonic) {
      R.rho = S(O.rho_bc[b]);
      R.p = (L.p + m.Pref) * pow(R.rho / L.rho, m.gamma) - m.Pref;
      R.T = m.temp(R.p, R.rho);
      R.a = sqrt(m.gamma * (R.p + m.Pref) / R.rho);
      R.V = L.V;
    } else {
      // everything extrapolated; R.rho keeps whatever the state cache held
      R.p = L.p; R.T = L.T; R.V = L.V;
    }
    if (MachL < 0.) {
      if (r.kind == DAMP_REVERSE) {
        R.p -= 0.5 * L.rho * uNL * uNL;
        R.rho = L.rho * pow((R.p + m.Pref), 1. / m.gamma) / pow((L.p + m.Pref), 1. / m.gamma);
        R.a = sqrt(m.gamma * (R.p + m.Pref) / R.rho);
        R.T = m.temp(R.p, R.rho);
      }
      if (r.kind == NO_REVERSE) R.V = vscale(-1., L.V);
    }
    if (MachL < 1. && r.kind == FORCE_SUPERSONIC) {
      R.p -= 0.5 * L.rho * pow(L.a - uNL, 2.);
      R.p = smin(S(1.e-8), R.p + m.Pref) - m.Pref;
      R.rho = L.rho * pow((R.p + m.Pref), 1. / m.gamma) / pow((L.p + m.Pref), 1. / m.gamma);
      R.a = sqrt(m.gamma * (R.p + m.Pref) / R.rho);
      R.T = m.temp(R.p, R.rho);
    }
  }
  void wall(CellState<S> &L, CellState<S> &R, bool is_slip) {
    const Material &m = O.material;
    int b = face.bc;
    if (O.bc[b].thermalType == FIXED_T) {
      R.T = R.T_center = S(O.T_bc[b]);
      R.p = L.p;
      R.rho = m.rho(R.p, R.T);
    } else {
      R.p = L.p; R.rho = L.rho; R.T = L.T; R.T_center = L.T_center;
    }
    if (is_slip) {
      R.V = vsub(L.V, vscale(2. * vdot(L.V, face.normal), face.normal));
      R.V_center = vsub(L.V_center, vscale(2. * vdot(L.V_center, face.normal), face.normal));
    } else {
      R.V = vscale(-1., L.V);
      R.V_center = vscale(-1., L.V_center);
    }
    R.p_center = L.p_center;
  }
  void symmetry(CellState<S> &L, CellState<S> &R) {
    R.p = L.p;
    R.V = vsub(L.V, vscale(2. * vdot(L.V, face.normal), face.normal));
    R.T = L.T;
    R.rho = L.rho;
    R.p_center = L.p_center;
    R.T_center = L.T_center;
    R.V_center = vsub(L.V_center, vscale(2. * vdot(L.V_center, face.normal), face.normal));
  }

  // ns_assemble_linear_system.cc:353-415
  void face_state_update(CellState<S> &L, CellState<S> &R) {
    if (face.bc >= 0) {
      face.gradu = F.gradu[face.parent]; face.gradv = F.gradv[face.parent];
      face.gradw = F.gradw[face.parent]; face.gradT = F.gradT[face.parent];
    } else {
      face.gradu = face_vec(F.gradu, face.index); face.gradv = face_vec(F.gradv, face.index);
      face.gradw = face_vec(F.gradw, face.index); face.gradT = face_vec(F.gradT, face.index);
    }
    Vec3 l2rnormal = face.left2right;
    l2rnormal = l2rnormal.norm();
    double l2rmag = fabs(face.left2right);
    auto corr = [&](V3<S> &gr, const S &d) {
      gr = vsub(gr, vscale(vdot(gr, l2rnormal), l2rnormal));
      gr = vadd(gr, vscale(d / l2rmag, l2rnormal));
    };
    corr(face.gradu, R.V_center[0] - L.V_center[0]);
    corr(face.gradv, R.V_center[1] - L.V_center[1]);
    corr(face.gradw, R.V_center[2] - L.V_center[2]);
    corr(face.gradT, R.T_center - L.T_center);
    face.V = vscale(0.5, vadd(L.V, R.V));
    face.T = 0.5 * (L.T + R.T);
    face.mu = O.material.viscosity(face.T);
    face.lambda = O.material.therm_cond(face.T);
  }

  // ns_roe.cc:25-98
  void roe_flux(CellState<S> &L, CellState<S> &R, S fn[5], S &wL) {
    double Gamma = O.material.gamma;
    S rho = sqrt(R.rho / L.rho);
    S u = (L.Vn[0] + rho * R.Vn[0]) / (1. + rho);
    S v = (L.Vn[1] + rho * R.Vn[1]) / (1. + rho);
    S w = (L.Vn[2] + rho * R.Vn[2]) / (1. + rho);
    S H = (L.H + rho * R.H) / (1. + rho);
    S a = sqrt((Gamma - 1.) * (H - 0.5 * (u * u + v * v + w * w)));
    rho *= L.rho;
    S Du = R.Vn[0] - L.Vn[0];
    S Dp = R.p - L.p;
    S deltaV, lambda, Dlambda, mdot, product;
    if (u >= 0.) {
      deltaV = 0.5 * (Dp - rho * a * Du) / (a * a);
      lambda = u - a;
      Dlambda = 2. * (smin(a, smax(S(0.), 2. * (L.a - R.a + Du))));
      if (lambda <= (-0.5 * Dlambda)) {
      } else if (lambda < (0.5 * Dlambda)) {
        lambda = -0.5 * (lambda - 0.5 * Dlambda) * (lambda - 0.5 * Dlambda) / Dlambda;
      } else {
        lambda = S(0.);
      }
      mdot = L.rho * L.Vn[0];
      product = lambda * deltaV;
      fn[0] = mdot + product;
      fn[1] = mdot * L.Vn[0] + L.p + product * (u - a);
      fn[2] = mdot * L.Vn[1] + product * v;
      fn[3] = mdot * L.Vn[2] + product * w;
      fn[4] = mdot * L.H + product * (H - u * a);
    } else {
      deltaV = 0.5 * (Dp + rho * a * Du) / (a * a);
      lambda = u + a;
      Dlambda = 2. * (smin(a, smax(S(0.), 2. * (R.a - L.a + Du))));
      if (lambda >= (0.5 * Dlambda)) {
      } else if (lambda > (-0.5 * Dlambda)) {
        lambda = 0.5 * (lambda + 0.5 * Dlambda) * (lambda + 0.5 * Dlambda) / Dlambda;
      } else {
        lambda = S(0.);
      }
      mdot = R.rho * R.Vn[0];
      product = lambda * deltaV;
      fn[0] = mdot - product;
      fn[1] = mdot * R.Vn[0] + R.p - product * (u + a);
      fn[2] = mdot * R.Vn[1] - product * v;
      fn[3] = mdot * R.Vn[2] - product * w;
      fn[4] = mdot * R.H - product * (H + u * a);
    }
    wL = S(0.5);
  }

  // ns_ausm_plus_up.cc:35-153
  static S M2p(const S &M) { return 0.25 * (M + 1.) * (M + 1.); }
  static S M2m(const S &M) { return -0.25 * (M - 1.) * (M - 1.); }
  static S M4p(const S &M, double beta) { if (fabs(M) >= 1.) return 0.5 * (M + fabs(M)); return M2p(M) * (1. - 16. * beta * M2m(M)); }
  static S M4m(const S &M, double beta) { if (fabs(M) >= 1.) return 0.5 * (M - fabs(M)); return M2m(M) * (1. + 16. * beta * M2p(M)); }
  static S P5p(const S &M, const S &alpha) { if (fabs(M) >= 1.) return 0.5 * (M + fabs(M)) / M; return M2p(M) * ((2. - M) - 16. * alpha * M * M2m(M)); }
  static S P5m(const S &M, const S &alpha) { if (fabs(M) >= 1.) return 0.5 * (M - fabs(M)) / M; return M2m(M) * ((-2. - M) + 16. * alpha * M * M2p(M)); }
  void ausm_flux(CellState<S> &L, CellState<S> &R, S fn[5], S &wL) {
    const double beta = 0.125, Kp = 0.25, Ku = 0.75, sigma = 1.;
    double Pref = O.material.Pref, Minf = O.Minf;
    S aL_star = L.a, aR_star = R.a;
    S aL_hat = aL_star * aL_star / smax(aL_star, L.Vn[0]);
    S aR_hat = aR_star * aR_star / smax(aR_star, -1. * R.Vn[0]);
    S a = smin(aL_hat, aR_hat);
    S rho = 0.5 * (L.rho + R.rho);
    S ML = L.Vn[0] / a;
    S MR = R.Vn[0] / a;
    S Mbar2 = 0.5 * (ML * ML + MR * MR);
    S Mref = smax(S(Minf), sqrt(Mbar2));
    Mref = smin(Mref, 1.);
    S fa;
    if (Mbar2 >= 1.) fa = S(1.);
    else {
      S Mo = sqrt(smin(S(1.), smax(Mbar2, Mref * Mref)));
      fa = Mo * (2. - Mo);
    }
    S M = M4p(ML, beta) + M4m(MR, beta) - Kp / fa * smax(1. - sigma * Mbar2, 0.) * (R.p - L.p) / (rho * a * a);
    S mdot;
    if (M > 0.) mdot = a * M * L.rho;
    else mdot = a * M * R.rho;
    S alpha = 3. / 16. * (-4. + 5. * fa * fa);
    S p = P5p(ML, alpha) * (L.p + Pref) + P5m(MR, alpha) * (R.p + Pref) -
          Ku * P5p(ML, alpha) * P5m(MR, alpha) * (L.rho + R.rho) * fa * a * (R.Vn[0] - L.Vn[0]);
    p -= Pref;
    fn[0] = mdot;
    if (mdot > 0.) {
      fn[1] = mdot * L.Vn[0] + p; fn[2] = mdot * L.Vn[1]; fn[3] = mdot * L.Vn[2]; fn[4] = mdot * L.H; wL = S(1.);
    } else {
      fn[1] = mdot * R.Vn[0] + p; fn[2] = mdot * R.Vn[1]; fn[3] = mdot * R.Vn[2]; fn[4] = mdot * R.H; wL = S(0.);
    }
  }

  // ns_sd_slau.cc:37-94, term by term (Csd1 = 0.1, Csd2 = 10, alpha = 0;
  // max_delta_p = |delta_p| as at ns_sd_slau.cc:64)
  static double signum(const S &x) { double r = re_(x); return double((r > 0) - (r < 0)); }
  void sdslau_flux(CellState<S> &L, CellState<S> &R, S fn[5], S &wL) {
    const double Csd1 = 0.1, Csd2 = 10., Pref = O.material.Pref;
    S a = 0.5 * (L.a + R.a);
    S LV2 = L.V[0] * L.V[0] + L.V[1] * L.V[1] + L.V[2] * L.V[2];
    S RV2 = R.V[0] * R.V[0] + R.V[1] * R.V[1] + R.V[2] * R.V[2];
    S Mhat = smin(S(1.), S(sqrt(0.5 * (LV2 + RV2) / a)));
    S chi = (1. - Mhat) * (1. - Mhat);
    S Mplus = L.Vn[0] / a;
    S Mminus = R.Vn[0] / a;
    S Bplus, Bminus;
    double alpha = 3. / 16. * (-4. + 5. * 0. * 0.);
    alpha = 0.;
    if (fabs(Mplus) < 1.) Bplus = 0.25 * (2. - Mplus) * (Mplus + 1.) * (Mplus + 1.) + alpha * Mplus * (Mplus - 1.) * (Mplus - 1.);
    else Bplus = S(0.5 * (1. + signum(Mplus)));
    if (fabs(Mminus) < 1.) Bminus = 0.25 * (2. + Mminus) * (Mminus - 1.) * (Mminus - 1.) - alpha * Mminus * (Mminus - 1.) * (Mminus - 1.);
    else Bminus = S(0.5 * (1. + signum(-1. * Mminus)));
    S ave_p = 0.5 * (L.p + R.p) + Pref;
    S delta_p = R.p - L.p;
    S p = ave_p - 0.5 * (Bplus - Bminus) * delta_p + (1. - chi) * (Bplus + Bminus - 1.) * ave_p;
    S max_delta_p = fabs(delta_p);
    S g = -1. * smax(smin(Mplus, S(0.)), S(-1.)) * smin(smax(Mminus, S(0.)), S(1.));
    S Vn = (L.rho * fabs(L.Vn[0]) + R.rho * fabs(R.Vn[0])) / (L.rho + R.rho);
    S Vnplus = (1. - g) * Vn + g * fabs(L.Vn[0]);
    S Vnminus = (1. - g) * Vn + g * fabs(R.Vn[0]);
    S theta = (Csd2 * fabs(delta_p) / ave_p + Csd1) / (max_delta_p / ave_p + Csd1);
    theta = smin(S(1.), S(theta * theta));
    S mdot = 0.5 * (L.rho * (L.Vn[0] + Vnplus) + R.rho * (R.Vn[0] - Vnminus) - theta * smax(S(0.), S(1. - Vn / a)) * delta_p / a);
    p -= Pref;
    fn[0] = mdot;
    if (mdot > 0.) {
      fn[1] = mdot * L.Vn[0] + p; fn[2] = mdot * L.Vn[1]; fn[3] = mdot * L.Vn[2]; fn[4] = mdot * L.H; wL = S(1.);
    } else {
      fn[1] = mdot * R.Vn[0] + p; fn[2] = mdot * R.Vn[1]; fn[3] = mdot * R.Vn[2]; fn[4] = mdot * R.H; wL = S(0.);
    }
  }

  // sqrt whose complex-step tangent is 0 where the value is 0 (the kink of
  // |x| at 0); the value is sqrt's
  static S sqrt0(const S &q) { return re_(q) == 0. ? S(0.) : S(sqrt(q)); }

  // ns_stegger_warming.cc:23-145, in the rotated frame with the explicit
  // 5x5 products: Jacob = (L diag(Lambda)) R per signal, flux += Jacob Q.
  void sw_flux(CellState<S> &L, CellState<S> &R, S fn[5], S &wL) {
    const Face &gf = O.grid.face[face.index];
    const double alpha = 6., RW = 8314.47215 / O.material.Mw, gam = O.material.gamma;
    const double Cp = O.material.Cp();
    const double beta = gam * RW / Cp;
    for (int i = 0; i < 5; ++i) fn[i] = S(0.);
    S deltap = fabs(L.p - R.p) / smin(L.p, R.p);
    S w = 0.5 / (alpha * alpha * deltap * deltap + 1.);
    for (int h = 0; h <= 1; ++h) {
      double signal = std::pow(-1., h);
      S weightL = (signal > 0.) ? S(1. - w) : w;
      S weightR = 1. - weightL;
      wL = weightL;
      S p = weightL * L.p + weightR * R.p;
      V3<S> V;
      for (int i = 0; i < 3; ++i) V[i] = weightL * L.Vn[i] + weightR * R.Vn[i];
      S V2 = sqrt0(V[0] * V[0] + V[1] * V[1] + V[2] * V[2]);
      S Vmag = V2;
      V2 = V2 * V2;
      S T = weightL * L.T + weightR * R.T;
      S rho = weightL * L.rho + weightR * R.rho;
      S a = sqrt((1. + beta) * p / rho);
      S a2 = a * a;
      S H = 0.5 * V2 + a2 / (gam - 1.);
      S gamma_s = RW * T + beta * (0.5 * V2 - Cp * T / gam);
      S eta = (beta * V2 - gamma_s) / (beta * a2);
      S Lm[5][5], Rm[5][5], Jac[5][5], Lam[5], Q[5];
      for (int i = 0; i < 5; ++i) for (int j = 0; j < 5; ++j) { Lm[i][j] = S(0.); Rm[i][j] = S(0.); }
      Lm[0][0] = 1.0 / a2;
      Lm[0][3] = 0.5 / a2; Lm[0][4] = 0.5 / a2;
      Lm[1][0] = V[0] / a2; Lm[2][0] = V[1] / a2; Lm[3][0] = V[2] / a2;
      Lm[1][3] = 0.5 * (V[0] + a) / a2;
      Lm[1][4] = 0.5 * (V[0] - a) / a2;
      Lm[2][1] = S(1.);
      Lm[2][3] = 0.5 * V[1] / a2; Lm[2][4] = Lm[2][3];
      Lm[3][2] = S(1.);
      Lm[3][3] = 0.5 * V[2] / a2; Lm[3][4] = Lm[3][3];
      Lm[4][0] = eta; Lm[4][1] = V[1]; Lm[4][2] = V[2];
      Lm[4][3] = 0.5 * (H + a * V[0]) / a2;
      Lm[4][4] = 0.5 * (H - a * V[0]) / a2;
      S eps;
      if (gf.closest_wall_distance > O.bl_height) eps = O.wdiss * (a + Vmag);
      else eps = O.wdiss * gf.dissipation_factor * (a + fabs(V[0]));
      Lam[0] = 0.5 * (V[0] + signal * sqrt0(V[0] * V[0] + eps * eps));
      Lam[1] = Lam[0]; Lam[2] = Lam[0];
      Lam[3] = 0.5 * (V[0] + a + signal * sqrt0((V[0] + a) * (V[0] + a) + eps * eps));
      Lam[4] = 0.5 * (V[0] - a + signal * sqrt0((V[0] - a) * (V[0] - a) + eps * eps));
      for (int i = 0; i < 5; ++i) for (int j = 0; j < 5; ++j) Lm[i][j] = Lm[i][j] * Lam[j];
      Rm[0][0] = a2 - gamma_s; Rm[0][1] = beta * V[0]; Rm[0][2] = beta * V[1]; Rm[0][3] = beta * V[2]; Rm[0][4] = S(-beta);
      Rm[1][0] = -1. * V[1]; Rm[1][2] = S(1.);
      Rm[2][0] = -1. * V[2]; Rm[2][3] = S(1.);
      Rm[3][0] = gamma_s - V[0] * a; Rm[3][1] = a - beta * V[0]; Rm[3][2] = -beta * V[1]; Rm[3][3] = -beta * V[2];
      Rm[4][0] = gamma_s + V[0] * a; Rm[4][1] = -1. * a - beta * V[0]; Rm[4][2] = -beta * V[1]; Rm[4][3] = -beta * V[2];
      Rm[3][4] = S(beta); Rm[4][4] = S(beta);
      for (int i = 0; i < 5; ++i)
        for (int j = 0; j < 5; ++j) {
          Jac[i][j] = S(0.);
          for (int k = 0; k < 5; ++k) Jac[i][j] += Lm[i][k] * Rm[k][j];
        }
      CellState<S> &U = (signal > 0.) ? L : R;
      Q[0] = U.rho;
      Q[1] = U.rho * U.Vn[0]; Q[2] = U.rho * U.Vn[1]; Q[3] = U.rho * U.Vn[2];
      Q[4] = U.rho * U.H - U.p;
      for (int i = 0; i < 5; ++i) for (int j = 0; j < 5; ++j) fn[i] += Jac[i][j] * Q[j];
    }
  }

  // ns_vanleer.cc:25-66
  void vanleer_flux(CellState<S> &L, CellState<S> &R, S fn[5], S &wL) {
    double Gamma = O.material.gamma, Pref = O.material.Pref;
    S ML = L.Vn[0] / L.a;
    S MR = R.Vn[0] / R.a;
    S M = 0.5 * (ML + MR);
    if (M <= -1.) {
      S mdot = R.rho * R.Vn[0];
      fn[0] = mdot; fn[1] = mdot * R.Vn[0] + R.p; fn[2] = mdot * R.Vn[1]; fn[3] = mdot * R.Vn[2]; fn[4] = mdot * R.H; wL = S(0.);
    } else if (M >= 1.) {
      S mdot = L.rho * L.Vn[0];
      fn[0] = mdot; fn[1] = mdot * L.Vn[0] + L.p; fn[2] = mdot * L.Vn[1]; fn[3] = mdot * L.Vn[2]; fn[4] = mdot * L.H; wL = S(1.);
    } else {
      S fplus = 0.25 * L.rho * L.a * (ML + 1.) * (ML + 1.);
      S fminus = -0.25 * R.rho * R.a * (1. - MR) * (1. - MR);
      fn[0] = fplus + fminus;
      S termL = (2. * L.a / Gamma) * (0.5 * (Gamma - 1) * ML + 1.);
      S termR = (2. * R.a / Gamma) * (0.5 * (Gamma - 1) * MR - 1.);
      fn[1] = fplus * termL + fminus * termR - Pref;
      fn[2] = fplus * L.Vn[1] + fminus * R.Vn[1];
      fn[3] = fplus * L.Vn[2] + fminus * R.Vn[2];
      termL = 0.5 * Gamma * Gamma / (Gamma * Gamma - 1.) * termL * termL + 0.5 * (L.Vn[1] * L.Vn[1] + L.Vn[2] * L.Vn[2]);
      termR = 0.5 * Gamma * Gamma / (Gamma * Gamma - 1.) * termR * termR + 0.5 * (R.Vn[1] * R.Vn[1] + R.Vn[2] * R.Vn[2]);
      fn[4] = fplus * termL + fminus * termR;
      wL = S(0.5);
    }
  }

  // ns_convective_face_flux.cc:32-59
  void convective_face_flux(CellState<S> &L, CellState<S> &R, S flux[5]) {
    S fn[5];
    S &wL = F.weightL[face.index];
    if (O.flux == ROE) roe_flux(L, R, fn, wL);
    else if (O.flux == VAN_LEER) vanleer_flux(L, R, fn, wL);
    else if (O.flux == SD_SLAU) sdslau_flux(L, R, fn, wL);
    else if (O.flux == SW) sw_flux(L, R, fn, wL);
    else ausm_flux(L, R, fn, wL);
    const Vec3 &n = face.normal, &t1 = face.tangent1, &t2 = face.tangent2;
    flux[0] = fn[0] * face.area;
    flux[1] = (fn[1] * n[0] + fn[2] * t1[0] + fn[3] * t2[0]) * face.area;
    flux[2] = (fn[1] * n[1] + fn[2] * t1[1] + fn[3] * t2[1]) * face.area;
    flux[3] = (fn[1] * n[2] + fn[2] * t1[2] + fn[3] * t2[2]) * face.area;
    flux[4] = fn[4] * face.area;
  }

  // ns_diffusive_face_flux.cc:28-64 (laminar; turbulent terms enter through mu_t)
  void diffusive_face_flux(S flux[5], const S &turb_visc, const S &turb_cond) {
    Vec3 areaVec = face.normal * face.area;
    V3<S> tx, ty, tz;
    const V3<S> &gu = face.gradu, &gv = face.gradv, &gw = face.gradw;
    tx[0] = 2. / 3. * (2. * gu[0] - gv[1] - gw[2]);
    tx[1] = gu[1] + gv[0];
    tx[2] = gu[2] + gw[0];
    ty[0] = tx[1];
    ty[1] = 2. / 3. * (2. * gv[1] - gu[0] - gw[2]);
    ty[2] = gv[2] + gw[1];
    tz[0] = tx[2];
    tz[1] = ty[2];
    tz[2] = 2. / 3. * (2. * gw[2] - gu[0] - gv[1]);
    S mu = face.mu + turb_visc;
    flux[1] = mu * vdot(tx, areaVec);
    flux[2] = mu * vdot(ty, areaVec);
    flux[3] = mu * vdot(tz, areaVec);
    flux[4] = mu * (vdot(tx, face.V) * areaVec[0] + vdot(ty, face.V) * areaVec[1] + vdot(tz, face.V) * areaVec[2]);
    S qq = (face.lambda + turb_cond) * vdot(face.gradT, areaVec);
    if (face.bc >= 0 && O.bc[face.bc].thermalType == FIXED_Q) qq = S(O.qdot_bc[face.bc] * face.area);
    flux[4] += qq;
  }

  // Reconstruction of the missing NavierStokes::update_boundaries: for every
  // boundary face (in face order) run face_geom_update, left_state_update with
  // ZERO gradients (the state right after initialise, ns.cc:93) and
  // right_state_update/apply_bcs, then store right.{p,V,T} in the ghost and
  // rho = EOS(p,T).  ghost_mode 1 stores the same BC state (identical values:
  // with zero gradients the left state is the cell-centre state).
  void update_boundaries() {
    Grid &g = O.grid;
    for (size_t c = 0; c < g.cell.size(); ++c) {
      F.gradp[c] = V3<S>(); F.gradu[c] = V3<S>(); F.gradv[c] = V3<S>(); F.gradw[c] = V3<S>(); F.gradT[c] = V3<S>();
    }
    CellState<S> L, R;
    for (int f = 0; f < g.faceCount; ++f) {
      if (g.face[f].bc < 0) continue;
      face_geom_update(f);
      left_state_update(L);
      right_state_update(L, R);
      int gh = g.face[f].neighbor;
      F.p[gh] = R.p;
      F.V[gh] = R.V;
      F.T[gh] = R.T;
      F.rho[gh] = O.material.rho(R.p, R.T);
    }
  }

  // ns_assemble_linear_system.cc:34-140 (residual part; no Jacobian)
  // loads: optional per-BC force and moment [bcCount][6], integrated as in
  // ns_assemble_linear_system.cc:108-119 (convective - diffusive momentum flux
  // of every face of the region; moment (x_f - moment center) x that flux)
  void assemble(std::vector<S> &rhs, const std::vector<S> *mu_t_face = nullptr, double Pr_t = 0.9,
                std::vector<S> *loads = nullptr) {
    Grid &g = O.grid;
    rhs.assign((size_t)g.cellCount * 5, S(0.));
    if (loads) loads->assign((size_t)g.bcCount * 6, S(0.));
    S fc[5], fd[5];
    for (int m = 0; m < 5; ++m) fd[m] = S(0.);
    for (int f = 0; f < g.faceCount; ++f) {
      int pa = g.face[f].parent, nb = g.face[f].neighbor;
      face_geom_update(f);
      left_state_update(left);
      right_state_update(left, right);
      face_state_update(left, right);
      convective_face_flux(left, right, fc);
      S tv(0.), tc(0.);
      if (mu_t_face) { tv = (*mu_t_face)[f]; tc = O.material.Cp() * tv / Pr_t; }
      diffusive_face_flux(fd, tv, tc);
      F.mdot[f] = (fc[0] - fd[0]) / face.area;
      if (loads && g.face[f].bc >= 0) {
        S t[3];
        for (int i = 0; i < 3; ++i) t[i] = fc[i + 1] - fd[i + 1];
        const Vec3 r = g.face[f].centroid - O.moment_center;
        S *L = &(*loads)[(size_t)g.face[f].bc * 6];
        for (int i = 0; i < 3; ++i) L[i] += t[i];
        L[3] += r[1] * t[2] - r[2] * t[1];
        L[4] += r[2] * t[0] - r[0] * t[2];
        L[5] += r[0] * t[1] - r[1] * t[0];
      }
      for (int i = 0; i < 5; ++i) {
        S value = fd[i] - fc[i] + S(0.);
        rhs[(size_t)pa * 5 + i] += value;
        if (g.face[f].bc == INTERNAL_FACE) {
          S v2 = -1. * (fd[i] - fc[i]) + S(0.);
          rhs[(size_t)nb * 5 + i] += v2;
        }
      }
    }
  }
};

// ---------------------------------------------------------------- RANS k-omega (rans_*.cc)

// RANS::set_bcs (rans_set_bcs.cc:25-83) with the NS face values it reads at
// initialisation (uniform IC state, NS ghosts updated), and the turbulence
// deck options (rans.cc:51-71).  Only model=k-omega is restated.
static void setup_rans(Oracle &O) {
  Section &g = O.input.section("grid", 0);
  Subsection &ts = g.sub("turbulence");
  O.turbulent = ts.is_found;
  if (!O.turbulent) return;
  if (ts.gs("model").value != "k-omega") throw DeckError("only the k-omega turbulence model is restated");
  O.kLow = ts.gd("klowlimit").value; O.kHigh = ts.gd("khighlimit").value;
  O.omegaLow = ts.gd("omegalowlimit").value; O.ratioLimit = ts.gd("viscosityratiolimit").value;
  O.Pr_t = ts.gd("turbulentPr").value;
  Grid &gr = O.grid;
  const Material &m = O.material;
  // uniform initial state of IC_1 (two of p, T, rho)
  Subsection &ic = g.sub("IC", 0);
  double p = ic.gd("p").value, T = ic.gd("T").value, rho = ic.gd("rho").value;
  if (ic.gd("p").is_found && ic.gd("rho").is_found) T = m.temp(p, rho);
  else if (ic.gd("rho").is_found && ic.gd("T").is_found) p = m.pres(rho, T);
  const V3d &icv = ic.gv("V").value;
  Fields<double> F;
  F.alloc(gr.cell.size(), (size_t)gr.faceCount);
  for (int c = 0; c < gr.cellCount; ++c) {
    F.p[c] = p; F.T[c] = T; F.V[c] = V3<double>(icv.c[0], icv.c[1], icv.c[2]); F.rho[c] = m.rho(p, T);
  }
  NS<double> ns(O, F);
  ns.update_boundaries();
  const int count = g.sub("BC", 0).count;
  O.kw_fixed.assign(count, 0); O.mut_fixed.assign(count, 0);
  O.k_bc.assign(count, 0.); O.omega_bc.assign(count, 0.); O.mut_bc.assign(count, 0.);
  for (int b = 0; b < count; ++b) {
    Subsection &region = g.sub("BC", b);
    const std::string type = region.gs("type").value, kind = region.gs("kind").value;
    const double intensity = region.gd("turbulenceintensity").value, ratio = region.gd("eddyviscosityratio").value;
    if (type == "inlet") {
      int fid = 0;
      for (int f = 0; f < gr.faceCount; ++f)
        if (gr.face[f].bc == b) { fid = f; break; }
      // NS Variable face values (variable.h:134-147)
      double rf = 0., Tf = 0.;
      Vec3 Vf;
      if (O.rho_fixed[b] && gr.face[fid].bc == b) rf = O.rho_bc[b];
      else for (auto &kv : gr.face[fid].average) rf += kv.second * F.rho[kv.first];
      Tf = ns.face_scalar(F.T, fid, 1);
      if (O.V_fixed[b] && gr.face[fid].bc == b) Vf = O.V_bc[b];
      else for (auto &kv : gr.face[fid].average)
        for (int i = 0; i < 3; ++i) Vf[i] += kv.second * F.V[kv.first][i];
      O.kw_fixed[b] = 1;
      double kb = intensity * fabs(Vf);
      kb *= 1.5 * kb;
      kb = std::max(O.kLow, kb);
      O.k_bc[b] = kb;
      O.omega_bc[b] = rf * kb / (ratio * m.viscosity(Tf));
      O.mut_fixed[b] = 1;
      O.mut_bc[b] = ratio * m.viscosity(Tf);
    } else if (type == "wall") {
      if (kind != "slip") { O.mut_fixed[b] = 1; O.mut_bc[b] = 0.; }
    }
  }
}

// RANS residual for the state (W, K): NS residual with the eddy viscosity,
// then RANS::terms (rans_terms.cc:39-275) right-hand side.  Ghost k, omega:
// the BC value where fixed on the BC, else the parent value (the missing
// RANS update_boundaries, reconstructed like the NS one).
template <class S>
static void rans_residual(Oracle &O, Fields<S> &F, const std::vector<S> &k, const std::vector<S> &om,
                          std::vector<S> &rhs_ns, std::vector<S> &rhs_k) {
  Grid &g = O.grid;
  const Material &m = O.material;
  NS<S> ns(O, F);
  ns.update_boundaries();
  ns.calc_cell_grads();
  ns.calc_limiter();
  const size_t nt = g.cell.size();
  std::vector<S> K(nt), Om(nt), mut(nt);
  for (int c = 0; c < g.cellCount; ++c) { K[c] = k[c]; Om[c] = om[c]; }
  for (int f = 0; f < g.faceCount; ++f) {
    const int b = g.face[f].bc;
    if (b < 0) continue;
    const int gh = g.face[f].neighbor, pa = g.face[f].parent;
    if (O.kw_fixed[b]) { K[gh] = S(O.k_bc[b]); Om[gh] = S(O.omega_bc[b]); }
    else { K[gh] = K[pa]; Om[gh] = Om[pa]; }
  }
  // rans_update_eddy_viscosity.cc:26-56 (k-omega branch), every cell
  for (size_t c = 0; c < nt; ++c) {
    S mu = m.viscosity(F.T[c]);
    mut[c] = F.rho[c] * K[c] / Om[c];
    mut[c] = smin(S(O.ratioLimit * mu), mut[c]);
  }
  // mu_t.face (variable.h:134-147)
  std::vector<S> mutf((size_t)g.faceCount);
  for (int f = 0; f < g.faceCount; ++f) {
    const int b = g.face[f].bc;
    if (b >= 0 && O.mut_fixed[b]) { mutf[f] = S(O.mut_bc[b]); continue; }
    S t(0.);
    for (auto &kv : g.face[f].average) t += kv.second * mut[kv.first];
    mutf[f] = t;
  }
  ns.assemble(rhs_ns, &mutf, O.Pr_t);
  // RANS::calc_cell_grads (rans.cc:167-173): interior cells; ghosts keep zero
  std::vector<V3<S>> gk(nt), go(nt);
  for (int c = 0; c < g.cellCount; ++c) { gk[c] = ns.scalar_gradient(K, c); go[c] = ns.scalar_gradient(Om, c); }
  rhs_k.assign((size_t)g.cellCount * 2, S(0.));
  typedef KOmega KW;
  for (int f = 0; f < g.faceCount; ++f) {
    const int pa = g.face[f].parent, nb = g.face[f].neighbor, b = g.face[f].bc;
    const S lam = m.viscosity(ns.face_scalar(F.T, f, 1));
    const S turb = mutf[f];
    const S md = F.mdot[f], wL = F.weightL[f], wR = 1. - wL;
    // get_kOmega (rans_terms.cc:277-319)
    const S kL = K[pa], oL = Om[pa], kR = K[nb], oR = Om[nb];
    V3<S> fgk, fgo;
    if (b >= 0) { fgk = gk[pa]; fgo = go[pa]; }
    else { fgk = ns.face_vec(gk, f); fgo = ns.face_vec(go, f); }
    Vec3 l2r = g.cell[nb].centroid - g.cell[pa].centroid;
    Vec3 e = l2r.norm();
    const double l2rmag = fabs(l2r);
    {
      S d = vdot(fgk, e);
      fgk = vsub(fgk, vscale(d, e));
      fgk = vadd(fgk, vscale((kR - kL) / l2rmag, e));
      S d2 = vdot(fgo, e);
      fgo = vsub(fgo, vscale(d2, e));
      fgo = vadd(fgo, vscale((oR - oL) / l2rmag, e));
    }
    const double A = g.face[f].area;
    S conv[2], diff[2];
    conv[0] = md * (wL * kL + wR * kR) * A;
    conv[1] = md * (wL * oL + wR * oR) * A;
    diff[0] = (lam + turb * KW::sigma_k) * vdot(fgk, g.face[f].normal) * A;
    diff[1] = (lam + turb * KW::sigma_omega) * vdot(fgo, g.face[f].normal) * A;
    for (int i = 0; i < 2; ++i) {
      S value = diff[i] - conv[i];
      rhs_k[(size_t)pa * 2 + i] += value;
      if (b < 0) { value = value * -1.; rhs_k[(size_t)nb * 2 + i] += value; }
    }
  }
  for (int c = 0; c < g.cellCount; ++c) {
    const V3<S> &gu = F.gradu[c], &gv = F.gradv[c], &gw = F.gradw[c];
    const S dudx = gu[0], dudy = gu[1], dudz = gu[2], dvdx = gv[0], dvdy = gv[1], dvdz = gv[2];
    const S dwdx = gw[0], dwdy = gw[1], dwdz = gw[2];
    const S divU = dudx + dvdy + dwdz;
    const S sr = sqrt(2. * (dudx * dudx + dvdy * dvdy + dwdz * dwdz) + (dudy + dvdx) * (dudy + dvdx) +
                      (dudz + dwdx) * (dudz + dwdx) + (dvdz + dwdy) * (dvdz + dwdy));
    S Prod = mut[c] * (sr * sr - 2. / 3. * divU * divU) - 2. / 3. * F.rho[c] * K[c] * divU;
    const S Dest = KW::beta_star * F.rho[c] * Om[c] * K[c];
    Prod = smin(Prod, S(10. * Dest));
    S src0 = Prod;
    src0 -= Dest;
    S src1 = KW::alpha * F.rho[c] / mut[c] * Prod;
    src1 -= KW::beta * F.rho[c] * Om[c] * Om[c];
    const double vol = g.cell[c].volume;
    rhs_k[(size_t)c * 2] += src0 * vol;
    rhs_k[(size_t)c * 2 + 1] += src1 * vol;
  }
}

// time_step.cc:143-224 (CFL_LOCAL / CFL_MAX step sizes for one time level)
static void local_dt(Oracle &O, const double *W, double cfl, int mode, double *dt) {
  Grid &g = O.grid;
  const Material &m = O.material;
  if (mode == 0) {
    for (int c = 0; c < g.cellCount; ++c) {
      double p = W[5 * c], T = W[5 * c + 4];
      Vec3 V(W[5 * c + 1], W[5 * c + 2], W[5 * c + 3]);
      double a = m.a(p, T);
      dt[c] = cfl * g.cell[c].lengthScale / (fabs(V) + a);
    }
  } else {
    double cur = 1.e20;
    for (int c = 0; c < g.cellCount; ++c) {
      double p = W[5 * c], T = W[5 * c + 4];
      Vec3 V(W[5 * c + 1], W[5 * c + 2], W[5 * c + 3]);
      double a = m.a(p, T);
      cur = std::min(cur, cfl * g.cell[c].lengthScale / (fabs(V) + a));
    }
    for (int c = 0; c < g.cellCount; ++c) dt[c] = cur;
  }
}

struct Handle {
  Oracle O;
  Fields<double> F;
};

}  // namespace orc

using namespace orc;

extern "C" {

// Build the oracle from a deck file and a CELL-type raw mesh.
void *orc_create(const char *deck_path, int n_nodes, const double *xyz, int n_cells, const int *cidx, const int *conn,
                 int n_bc, const int *bc_index, const int *bc_nodes, char *err, int errlen) {
  auto H = std::make_unique<Handle>();
  try {
    Oracle &O = H->O;
    O.input.setFile(deck_path);
    register_deck_schema(O.input);
    std::string dp(deck_path);
    size_t slash = dp.find_last_of('/');
    std::string dir = (slash == std::string::npos) ? std::string() : dp.substr(0, slash);
    Grid &g = O.grid;
    g.bocoNodes.resize(n_bc);
    for (int b = 0; b < n_bc; ++b)
      for (int k = bc_index[b]; k < bc_index[b + 1]; ++k) g.bocoNodes[b].insert(bc_nodes[k]);
    create_nodes_cells(g, xyz, n_nodes, n_cells, cidx, conn);
    create_faces(g);
    g.bcCount = n_bc;
    areas_volumes(g);
    create_boundary_ghosts(g);
    set_bcs_global(O);
    setup_physics(O, dir);
    set_lengthScales(O);
    face_interpolation_weights(O);
    gradient_maps(O);
    H->F.alloc(g.cell.size(), (size_t)g.faceCount);
    setup_rans(O);
  } catch (const std::exception &e) {
    if (err && errlen > 0) { std::snprintf(err, errlen, "%s", e.what()); }
    return nullptr;
  }
  return H.release();
}

// Build the oracle from a deck file and a Tecplot FEPolyhedron grid file.
void *orc_create_tecplot(const char *deck_path, const char *grid_path, char *err, int errlen) {
  auto H = std::make_unique<Handle>();
  try {
    Oracle &O = H->O;
    O.input.setFile(deck_path);
    register_deck_schema(O.input);
    std::string dp(deck_path);
    size_t slash = dp.find_last_of('/');
    std::string dir = (slash == std::string::npos) ? std::string() : dp.substr(0, slash);
    Grid &g = O.grid;
    TecRaw raw = read_tec(grid_path);
    g.bocoNodes = raw.bocoNodes;
    std::map<int, int> g2l;
    create_nodes_cells(g, raw.xyz.data(), raw.nNodes, raw.nCells, raw.cellConnIndex.data(), raw.cellConnectivity.data(), &g2l);
    create_faces2(g, raw, g2l);
    g.bcCount = (int)raw.bocoNodes.size();
    areas_volumes(g);
    create_boundary_ghosts(g);
    set_bcs_global(O);
    setup_physics(O, dir);
    set_lengthScales(O);
    face_interpolation_weights(O);
    gradient_maps(O);
    H->F.alloc(g.cell.size(), (size_t)g.faceCount);
    setup_rans(O);
  } catch (const std::exception &e) {
    if (err && errlen > 0) { std::snprintf(err, errlen, "%s", e.what()); }
    return nullptr;
  }
  return H.release();
}

void orc_destroy(void *h) { delete static_cast<Handle *>(h); }

// sizes: [n_cells, n_faces, n_ghosts, n_total, n_nodes, stencil_entries, cell_face_entries, dimension]
void orc_sizes(void *h, long long *out) {
  Grid &g = static_cast<Handle *>(h)->O.grid;
  long long st = 0, cf = 0;
  for (int c = 0; c < g.cellCount; ++c) { st += (long long)g.cell[c].gradMap.size(); cf += (long long)g.cell[c].faces.size(); }
  out[0] = g.cellCount; out[1] = g.faceCount; out[2] = (long long)g.cell.size() - g.cellCount;
  out[3] = (long long)g.cell.size(); out[4] = g.nodeCount; out[5] = st; out[6] = cf; out[7] = g.dimension;
}

// Integer connectivity in reference order.
void orc_connectivity(void *h, int *face_parent, int *face_neighbor, int *face_bc, int *face_nodes /* nf*4, -1 pad */,
                      int *cell_face_index /* nc+1 */, int *cell_faces, int *nbr_index /* nc+1 */, int *nbrs,
                      int *grad_index /* nc+1 */, int *grad_keys) {
  Grid &g = static_cast<Handle *>(h)->O.grid;
  for (int f = 0; f < g.faceCount; ++f) {
    face_parent[f] = g.face[f].parent; face_neighbor[f] = g.face[f].neighbor; face_bc[f] = g.face[f].bc;
    for (int k = 0; k < 4; ++k) face_nodes[4 * f + k] = k < (int)g.face[f].nodes.size() ? g.face[f].nodes[k] : -1;
  }
  int a = 0, b = 0, c2 = 0;
  cell_face_index[0] = 0; nbr_index[0] = 0; grad_index[0] = 0;
  for (int c = 0; c < g.cellCount; ++c) {
    for (int f : g.cell[c].faces) cell_faces[a++] = f;
    for (int n : g.cell[c].neighborCells) nbrs[b++] = n;
    for (auto &kv : g.cell[c].gradMap) grad_keys[c2++] = kv.first;
    cell_face_index[c + 1] = a; nbr_index[c + 1] = b; grad_index[c + 1] = c2;
  }
}

int orc_nbr_total(void *h) {
  Grid &g = static_cast<Handle *>(h)->O.grid;
  long long t = 0;
  for (int c = 0; c < g.cellCount; ++c) t += (long long)g.cell[c].neighborCells.size();
  return (int)t;
}

// Geometry: face normal/area/centroid/avg weights, cell centroid/volume/lengthScale/wall distance (incl. ghosts)
void orc_geometry(void *h, double *fn, double *fa, double *fc, double *favg /* nf*2 (parent, neighbor) */,
                  double *cc, double *cv, double *cls, double *cwd, double *lref) {
  Grid &g = static_cast<Handle *>(h)->O.grid;
  for (int f = 0; f < g.faceCount; ++f) {
    for (int k = 0; k < 3; ++k) { fn[3 * f + k] = g.face[f].normal[k]; fc[3 * f + k] = g.face[f].centroid[k]; }
    fa[f] = g.face[f].area;
    auto &avg = g.face[f].average;
    favg[2 * f] = avg.count(g.face[f].parent) ? avg.at(g.face[f].parent) : 0.;
    favg[2 * f + 1] = avg.count(g.face[f].neighbor) ? avg.at(g.face[f].neighbor) : 0.;
  }
  for (size_t c = 0; c < g.cell.size(); ++c) {
    for (int k = 0; k < 3; ++k) cc[3 * c + k] = g.cell[c].centroid[k];
    cv[c] = g.cell[c].volume; cls[c] = g.cell[c].lengthScale; cwd[c] = g.cell[c].closest_wall_distance;
  }
  *lref = g.lengthScale;
}

// Gradient-map weights in map (ascending key) order, three doubles per entry.
void orc_grad_weights(void *h, double *w) {
  Grid &g = static_cast<Handle *>(h)->O.grid;
  size_t k = 0;
  for (int c = 0; c < g.cellCount; ++c)
    for (auto &kv : g.cell[c].gradMap) { w[k++] = kv.second[0]; w[k++] = kv.second[1]; w[k++] = kv.second[2]; }
}

// FP64 residual of the interior-cell primitive state W[nc][5] = (p,u,v,w,T).
// Optional outputs (may be null): mdot[nf], weightL[nf], grads[ntot][15]
// (p,u,v,w,T gradients), limiter[nc][5], ghost[nghost][5].
int orc_residual(void *h, const double *W, double *R, double *mdot, double *weightL, double *grads, double *limiter,
                 double *ghost, char *err, int errlen) {
  Handle *H = static_cast<Handle *>(h);
  Oracle &O = H->O;
  Grid &g = O.grid;
  Fields<double> &F = H->F;
  try {
    for (int c = 0; c < g.cellCount; ++c) {
      F.p[c] = W[5 * c]; F.V[c] = V3<double>(W[5 * c + 1], W[5 * c + 2], W[5 * c + 3]); F.T[c] = W[5 * c + 4];
      F.rho[c] = O.material.rho(F.p[c], F.T[c]);
    }
    for (int i = 0; i < 5; ++i)
      for (size_t c = 0; c < g.cell.size(); ++c) F.limiter[i][c] = (O.order == FIRST) ? 0. : 1.;
    NS<double> ns(O, F);
    ns.update_boundaries();
    ns.calc_cell_grads();
    ns.calc_limiter();
    std::vector<double> rhs;
    ns.assemble(rhs);
    std::memcpy(R, rhs.data(), sizeof(double) * rhs.size());
    if (mdot) for (int f = 0; f < g.faceCount; ++f) mdot[f] = F.mdot[f];
    if (weightL) for (int f = 0; f < g.faceCount; ++f) weightL[f] = F.weightL[f];
    if (grads) {
      for (size_t c = 0; c < g.cell.size(); ++c) {
        const V3<double> *gs[5] = {&F.gradp[c], &F.gradu[c], &F.gradv[c], &F.gradw[c], &F.gradT[c]};
        for (int v = 0; v < 5; ++v) for (int k = 0; k < 3; ++k) grads[15 * c + 3 * v + k] = (*gs[v])[k];
      }
    }
    if (limiter) for (int c = 0; c < g.cellCount; ++c) for (int v = 0; v < 5; ++v) limiter[5 * c + v] = F.limiter[v][c];
    if (ghost) {
      for (size_t c = g.cellCount; c < g.cell.size(); ++c) {
        size_t k = c - g.cellCount;
        ghost[5 * k] = F.p[c]; ghost[5 * k + 1] = F.V[c][0]; ghost[5 * k + 2] = F.V[c][1];
        ghost[5 * k + 3] = F.V[c][2]; ghost[5 * k + 4] = F.T[c];
      }
    }
  } catch (const std::exception &e) {
    if (err && errlen > 0) std::snprintf(err, errlen, "%s", e.what());
    return 1;
  }
  return 0;
}

// Complex-step directional derivative: dR = Im(R(W + i*h*dW))/h.
int orc_residual_cstep(void *h, const double *W, const double *dW, double hstep, double *dR, char *err, int errlen) {
  Handle *H = static_cast<Handle *>(h);
  Oracle &O = H->O;
  Grid &g = O.grid;
  Fields<CStep> F;
  F.alloc(g.cell.size(), (size_t)g.faceCount);
  try {
    for (int c = 0; c < g.cellCount; ++c) {
      F.p[c] = CStep(W[5 * c], hstep * dW[5 * c]);
      F.V[c] = V3<CStep>(CStep(W[5 * c + 1], hstep * dW[5 * c + 1]), CStep(W[5 * c + 2], hstep * dW[5 * c + 2]),
                         CStep(W[5 * c + 3], hstep * dW[5 * c + 3]));
      F.T[c] = CStep(W[5 * c + 4], hstep * dW[5 * c + 4]);
      F.rho[c] = O.material.rho(F.p[c], F.T[c]);
    }
    for (int i = 0; i < 5; ++i)
      for (size_t c = 0; c < g.cell.size(); ++c) F.limiter[i][c] = CStep((O.order == FIRST) ? 0. : 1.);
    NS<CStep> ns(O, F);
    ns.update_boundaries();
    ns.calc_cell_grads();
    ns.calc_limiter();
    std::vector<CStep> rhs;
    ns.assemble(rhs);
    for (size_t k = 0; k < rhs.size(); ++k) dR[k] = rhs[k].im / hstep;
  } catch (const std::exception &e) {
    if (err && errlen > 0) std::snprintf(err, errlen, "%s", e.what());
    return 1;
  }
  return 0;
}

// RANS k-omega residual: R[nc][5] (NS with eddy viscosity) and RK[nc][2]
// for the state W[nc][5], K[nc][2] = (k, omega).
int orc_rans_residual(void *h, const double *W, const double *Kin, double *R, double *RK, char *err, int errlen) {
  Handle *H = static_cast<Handle *>(h);
  Oracle &O = H->O;
  Grid &g = O.grid;
  Fields<double> &F = H->F;
  try {
    if (!O.turbulent) throw DeckError("the deck has no turbulence section");
    for (int c = 0; c < g.cellCount; ++c) {
      F.p[c] = W[5 * c]; F.V[c] = V3<double>(W[5 * c + 1], W[5 * c + 2], W[5 * c + 3]); F.T[c] = W[5 * c + 4];
      F.rho[c] = O.material.rho(F.p[c], F.T[c]);
    }
    for (int i = 0; i < 5; ++i)
      for (size_t c = 0; c < g.cell.size(); ++c) F.limiter[i][c] = (O.order == FIRST) ? 0. : 1.;
    std::vector<double> k(g.cellCount), om(g.cellCount), rns, rk;
    for (int c = 0; c < g.cellCount; ++c) { k[c] = Kin[2 * c]; om[c] = Kin[2 * c + 1]; }
    rans_residual(O, F, k, om, rns, rk);
    std::memcpy(R, rns.data(), sizeof(double) * rns.size());
    std::memcpy(RK, rk.data(), sizeof(double) * rk.size());
  } catch (const std::exception &e) {
    if (err && errlen > 0) std::snprintf(err, errlen, "%s", e.what());
    return 1;
  }
  return 0;
}

// Complex-step directional derivative of the RANS residual along (dW, dK):
// dR[nc][5], dRK[nc][2].
int orc_rans_residual_cstep(void *h, const double *W, const double *Kin, const double *dW, const double *dK, double hstep,
                            double *dR, double *dRK, char *err, int errlen) {
  Handle *H = static_cast<Handle *>(h);
  Oracle &O = H->O;
  Grid &g = O.grid;
  Fields<CStep> F;
  F.alloc(g.cell.size(), (size_t)g.faceCount);
  try {
    if (!O.turbulent) throw DeckError("the deck has no turbulence section");
    for (int c = 0; c < g.cellCount; ++c) {
      auto at = [&](int k) { return CStep(W[5 * c + k], hstep * dW[5 * c + k]); };
      F.p[c] = at(0);
      F.V[c] = V3<CStep>(at(1), at(2), at(3));
      F.T[c] = at(4);
      F.rho[c] = O.material.rho(F.p[c], F.T[c]);
    }
    for (int i = 0; i < 5; ++i)
      for (size_t c = 0; c < g.cell.size(); ++c) F.limiter[i][c] = CStep((O.order == FIRST) ? 0. : 1.);
    std::vector<CStep> k(g.cellCount), om(g.cellCount), rns, rk;
    for (int c = 0; c < g.cellCount; ++c) {
      k[c] = CStep(Kin[2 * c], hstep * dK[2 * c]);
      om[c] = CStep(Kin[2 * c + 1], hstep * dK[2 * c + 1]);
    }
    rans_residual(O, F, k, om, rns, rk);
    for (size_t i = 0; i < rns.size(); ++i) dR[i] = rns[i].im / hstep;
    for (size_t i = 0; i < rk.size(); ++i) dRK[i] = rk[i].im / hstep;
  } catch (const std::exception &e) {
    if (err && errlen > 0) std::snprintf(err, errlen, "%s", e.what());
    return 1;
  }
  return 0;
}

// Fixed BC values of the RANS variables: per BC [kw_fixed, k, omega, mut_fixed, mu_t].
void orc_rans_bcs(void *h, double *out) {
  Oracle &O = static_cast<Handle *>(h)->O;
  for (size_t b = 0; b < O.kw_fixed.size(); ++b) {
    out[5 * b] = O.kw_fixed[b]; out[5 * b + 1] = O.k_bc[b]; out[5 * b + 2] = O.omega_bc[b];
    out[5 * b + 3] = O.mut_fixed[b]; out[5 * b + 4] = O.mut_bc[b];
  }
}

// Boundary loads: force[bcCount][3] (and, non-null, moment[bcCount][3] about
// the deck's moment center) for state W, and (dW non-null) their complex-step
// directional derivatives along dW instead.
int orc_loads(void *h, const double *W, const double *dW, double hstep, double *force, double *moment, char *err,
              int errlen) {
  Handle *H = static_cast<Handle *>(h);
  Oracle &O = H->O;
  Grid &g = O.grid;
  Fields<CStep> F;
  F.alloc(g.cell.size(), (size_t)g.faceCount);
  try {
    const double hs = dW ? hstep : 0.;
    for (int c = 0; c < g.cellCount; ++c) {
      auto at = [&](int k) { return CStep(W[5 * c + k], dW ? hs * dW[5 * c + k] : 0.); };
      F.p[c] = at(0);
      F.V[c] = V3<CStep>(at(1), at(2), at(3));
      F.T[c] = at(4);
      F.rho[c] = O.material.rho(F.p[c], F.T[c]);
    }
    for (int i = 0; i < 5; ++i)
      for (size_t c = 0; c < g.cell.size(); ++c) F.limiter[i][c] = CStep((O.order == FIRST) ? 0. : 1.);
    NS<CStep> ns(O, F);
    ns.update_boundaries();
    ns.calc_cell_grads();
    ns.calc_limiter();
    std::vector<CStep> rhs, loads;
    ns.assemble(rhs, nullptr, 0.9, &loads);
    for (int b = 0; b < g.bcCount; ++b)
      for (int i = 0; i < 3; ++i) {
        const CStep &fv = loads[(size_t)b * 6 + i], &mv = loads[(size_t)b * 6 + 3 + i];
        force[b * 3 + i] = dW ? fv.im / hstep : fv.re;
        if (moment) moment[b * 3 + i] = dW ? mv.im / hstep : mv.re;
      }
  } catch (const std::exception &e) {
    if (err && errlen > 0) std::snprintf(err, errlen, "%s", e.what());
    return 1;
  }
  return 0;
}

// Local time step (mode 0: CFL_LOCAL; mode 1: CFL_MAX global minimum).
void orc_local_dt(void *h, const double *W, double cfl, int mode, double *dt) {
  local_dt(static_cast<Handle *>(h)->O, W, cfl, mode, dt);
}

// NavierStokes::cons2prim (ns_time_terms.cc:26-56) and the dt part of
// NavierStokes::time_terms (ns_time_terms.cc:140-158, ps_step_max = 1): the
// diagonal block P[i][j] * volume / dt of cell c, blocks[c][5][5], for the
// state W[nc][5] and local time steps dt[nc].  rho = EOS(p, T) as
// update_variables (ns.cc:357) leaves it; Cp is the ideal-gas value.
void orc_time_terms(void *h, const double *W, const double *dt, double *blocks) {
  Oracle &O = static_cast<Handle *>(h)->O;
  const Grid &g = O.grid;
  const Material &m = O.material;
  for (int c = 0; c < g.cellCount; ++c) {
    const double p = W[5 * c], T = W[5 * c + 4];
    const Vec3 V(W[5 * c + 1], W[5 * c + 2], W[5 * c + 3]);
    const double rho = m.rho(p, T);
    const double pressure = p + m.Pref;
    const double temperature = T + m.Tref;
    const double drho_dT = -1. * rho / temperature;
    const double drho_dp = rho / pressure;
    const double c_p = m.Cp();
    const double H = c_p * temperature + 0.5 * (V[0] * V[0] + V[1] * V[1] + V[2] * V[2]);
    double P[5][5] = {{0.}};
    P[0][0] = drho_dp; P[0][4] = drho_dT;
    P[1][0] = drho_dp * V[0]; P[1][1] = rho; P[1][4] = drho_dT * V[0];
    P[2][0] = drho_dp * V[1]; P[2][2] = rho; P[2][4] = drho_dT * V[1];
    P[3][0] = drho_dp * V[2]; P[3][3] = rho; P[3][4] = drho_dT * V[2];
    P[4][0] = drho_dp * H - 1.;
    P[4][1] = rho * V[0];
    P[4][2] = rho * V[1];
    P[4][3] = rho * V[2];
    P[4][4] = drho_dT * H + rho * c_p;
    for (int i = 0; i < 5; ++i)
      for (int j = 0; j < 5; ++j) blocks[25 * (size_t)c + 5 * i + j] = P[i][j] * g.cell[c].volume / dt[c];
  }
}

// Parsed case summary (for deck-parser parity with the product):
// [gamma, R, Pref, Tref, Minf, limiter_threshold, mu, lambda, sut_mu_ref, sut_T_ref, sut_S, Pr, lengthScale]
// ints: [flux, limiter, order, sutherland, prandtl, n_bc, dimension] then per BC [type, kind, specified, thermalType]
void orc_case_summary(void *h, double *dv, int *iv) {
  Oracle &O = static_cast<Handle *>(h)->O;
  const Material &m = O.material;
  double d[] = {m.gamma, m.R, m.Pref, m.Tref, O.Minf, O.limiter_threshold, m.mu, m.lambda,
                m.sut_mu_ref, m.sut_T_ref, m.sut_S, m.Pr, O.grid.lengthScale};
  std::memcpy(dv, d, sizeof(d));
  iv[0] = O.flux; iv[1] = O.limiter_function; iv[2] = O.order; iv[3] = m.sutherland; iv[4] = m.prandtl;
  iv[5] = (int)O.bc.size(); iv[6] = O.grid.dimension;
  for (size_t b = 0; b < O.bc.size(); ++b) {
    iv[7 + 4 * b] = O.bc[b].type; iv[8 + 4 * b] = O.bc[b].kind; iv[9 + 4 * b] = O.bc[b].specified; iv[10 + 4 * b] = O.bc[b].thermalType;
  }
}

}  // extern "C"
