// ORACLE — TEST INFRASTRUCTURE ONLY.
//
// Driver for the reference itself: Free CFD's own, unmodified sources (every
// .cc under the reference's src/, compiled by oracle/Makefile against the
// single-process stand-ins in oracle/ref/include/) linked with this file into
// oracle/_ref/freecfd_ref.  It runs the reference's set-up sequence of
// main.cc:131-245 for one grid, then calls the reference's own member
// functions for the quantities the tests compare:
//
//   mesh      Grid::setup, set_bcs, set_lengthScales, face_interpolation_weights,
//             gradient_maps -> connectivity, geometry, LSQ weights
//   residual  NavierStokes::calc_cell_grads (ns.cc:301-336), calc_limiter
//             (ns_limiters.cc:26-248), assemble_linear_system
//             (ns_assemble_linear_system.cc:34-195) -> rhs Vec, mdot, weightL,
//             gradients, limiters, ghost states; with a k-omega state also
//             RANS::update_eddy_viscosity, calc_cell_grads and terms
//             (rans_terms.cc:39-275) -> the RANS rhs Vec
//   timeterms NavierStokes::time_terms (ns_time_terms.cc:107-186, cons2prim
//             26-56) -> the 5x5 diagonal blocks P V / dt it adds
//   diagblocks the diagonal blocks of the implicit operator: the
//             finite-difference face Jacobians of assemble_linear_system plus
//             time_terms' P V / dt
//   dt        update_time_step (time_step.cc:143-224) at time step 1
//   bench     a given number of residual evaluations, timed (CPU baseline)
//
// Five pieces are supplied here because the snapshot of the reference lacks
// them or they cannot compile or run as compiled today:
//   * NavierStokes::update_boundaries and RANS::update_boundaries: declared
//     (ns.h:165, rans.h) and called (ns.cc:93,113, rans.cc:76,93) but their
//     sources (ns_update_boundaries.cc, rans_update_boundaries.cc, listed in
//     the CMakeLists) are absent.  Reconstruction, the same one the oracle
//     restatement and the CUDA path use: for every boundary face in face
//     order, face_geom_update -> left_state_update with zero gradients (the
//     state at initialise, "grads are initialized to zero. This update will be
//     first order", ns.cc:93) -> right_state_update / apply_bcs; the ghost
//     takes right.{p,V,T} and rho = EOS(p,T).  RANS ghosts take the BC value
//     where k / omega are fixed on the BC, else the parent cell's value.
//   * HeatConduction::set_bcs (heat_conduction/hc_set_bcs.cc redeclares a
//     loop variable and is rejected by current compilers); heat conduction is
//     not on this path and the stub refuses to run.
//   * Grid::create_partition_ghosts (grid_create_elements.cc:561-700) has no
//     return statement, which current GCC compiles into a trap; its one-rank
//     branch is restated below and the link redirects the call to it.
//   * set_bcs (set_bcs.cc:71-83) leaves BCregion fields uninitialised; the
//     driver sets the ones it leaves unset to NONE right after it returns.
//   * Grid::read_raw (grid_reader_cgns.cc:433-489) does not set raw.type; the
//     raw file only ever holds cell-type data (Grid::write_raw, grid.cc:346-394),
//     so the driver sets CELL.
// Grids enter through the reference's own raw grid file "grid.raw" in the case
// directory (written by oracle/reference.py in Grid::write_raw's layout).
//
// Usage: freecfd_ref <case_dir> <deck_basename> <command> [args]
// Output files are raw native-endian doubles / int32; a line
// "FCFD_REF_RESULT <json>" on stdout carries sizes and timings.
#include <sys/time.h>
#include <unistd.h>

#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "ns.h"
#include "rans.h"
#include "hc.h"

// Defined by the reference's main.cc (compiled with main renamed).
extern InputFile input;
extern vector<Grid> grid;
extern vector<vector<BCregion> > bc;
extern vector<NavierStokes> ns;
extern vector<HeatConduction> hc;
extern vector<RANS> rans;
extern vector<bool> turbulent;
extern vector<Variable<double> > dt;
extern vector<int> equations;
extern vector<vector<BC_Interface> > interface;
extern vector<Loads> loads;
extern int Rank, np;

void read_inputs(void);
void set_bcs(int gid);
void set_lengthScales(int gid);
void face_interpolation_weights(int gid);
void node_interpolation_weights(int gid);
void gradient_maps(int gid);
void set_time_step_options(void);
void set_pseudo_time_step_options(void);
void update_time_step(int timeStep, double &time, double &max_cfl, int gid);

// Stand-in globals of the stub headers.
int fcfd_ref_mat_capture = 0;
int fcfd_ref_mat_cap_lo = 0, fcfd_ref_mat_cap_hi = 0;
static int fcfd_ref_petsc_print(const char[], ...) { return 0; }
int (*PetscErrorPrintf)(const char[], ...) = fcfd_ref_petsc_print;

// ---------------------------------------------------------------- reconstructions

void NavierStokes::update_boundaries(void) {
  Grid &g = grid[gid];
  for (size_t c = 0; c < g.cell.size(); ++c) {
    gradp.cell(c) = 0.; gradu.cell(c) = 0.; gradv.cell(c) = 0.; gradw.cell(c) = 0.; gradT.cell(c) = 0.;
  }
  order_factor = 1.;
  NS_Cell_State L = NS_Cell_State(), R = NS_Cell_State();
  NS_Face_State F = NS_Face_State();
  L.update.resize(5, 0.);
  R.update.resize(5, 0.);
  for (int f = 0; f < g.faceCount; ++f) {
    if (g.face[f].bc < 0) continue;
    face_geom_update(F, f);
    left_state_update(L, F);
    right_state_update(L, R, F);
    const int gh = g.face[f].neighbor;
    p.cell(gh) = R.p;
    V.cell(gh) = R.V;
    T.cell(gh) = R.T;
    rho.cell(gh) = material.rho(R.p, R.T);
  }
}

void RANS::update_boundaries(void) {
  Grid &g = grid[gid];
  for (int f = 0; f < g.faceCount; ++f) {
    const int b = g.face[f].bc;
    if (b < 0) continue;
    const int gh = g.face[f].neighbor, pa = g.face[f].parent;
    if (k.fixedonBC[b]) {
      k.cell(gh) = k.bc(b);
      omega.cell(gh) = omega.bc(b);
    } else {
      k.cell(gh) = k.cell(pa);
      omega.cell(gh) = omega.cell(pa);
    }
  }
}

// Grid::create_partition_ghosts (grid_create_elements.cc:561-700) for one
// rank.  The reference's function has no return statement, so current
// compilers end it with a trap; the link sends Grid::setup's call here.  With
// one rank the partition-ghost search (566-651) does not run, the
// neighbouring-ghost loop (653-676) finds no ghost (boundary ghosts are
// created later, in create_boundary_ghosts), and what remains is the face
// bookkeeping of 678-699.
extern "C" int __wrap__ZN4Grid23create_partition_ghostsEv(Grid *g) {
  if (g->np != 1) throw std::runtime_error("the single-process reference build has one rank");
  g->globalNumFaceNodes = 0;
  g->globalFaceCount = 0;
  for (int f = 0; f < g->faceCount; ++f) {
    g->globalNumFaceNodes += (int)g->face[f].nodes.size();
    g->globalFaceCount++;
  }
  g->partition_ghosts_begin = g->cellCount;
  g->partition_ghosts_end = (int)g->cell.size() - 1;
  return 0;
}

// set_bcs (set_bcs.cc:71-83) builds each BCregion in an uninitialised local
// and sets only type (and kind = SLIP for slip walls); NavierStokes::set_bcs
// (ns_set_bcs.cc) later sets specified / thermalType / kind only where the
// deck gives them, so the reference reads indeterminate values for the rest.
// The oracle and the CUDA path read those as NONE ("not specified").  Right
// after set_bcs returns, before anything reads them, the driver gives the
// fields set_bcs.cc left unset that value; check_bc_fields then confirms every
// field holds NONE or a value the reference defines.
static void define_unset_bc_fields(int gid) {
  for (size_t b = 0; b < bc[gid].size(); ++b) {
    BCregion &r = bc[gid][b];
    const std::string kind = input.section("grid", gid).subsection("BC", (int)b).get_string("kind");
    if (kind != "slip") r.kind = NONE;
    r.specified = NONE;
    r.thermalType = NONE;
  }
}

static void check_bc_fields(int gid) {
  for (size_t b = 0; b < bc[gid].size(); ++b) {
    const BCregion &r = bc[gid][b];
    const bool kind_ok = r.kind == NONE || (r.kind >= NO_REVERSE && r.kind <= FORCE_SUPERSONIC);
    const bool spec_ok = r.specified == NONE || (r.specified >= BC_RHO && r.specified <= BC_V);
    const bool th_ok = r.thermalType == NONE || (r.thermalType >= FIXED_T && r.thermalType <= ADIABATIC);
    if (!kind_ok || !spec_ok || !th_ok) {
      std::ostringstream m;
      m << "BC_" << b + 1 << " holds an indeterminate field (kind " << r.kind << ", specified " << r.specified
        << ", thermalType " << r.thermalType << ")";
      throw std::runtime_error(m.str());
    }
  }
}

void HeatConduction::set_bcs(void) {
  throw std::runtime_error("heat conduction is not part of this build of the reference");
}

// ---------------------------------------------------------------- file helpers

template <class T>
static std::vector<T> read_bin(const std::string &path, size_t n) {
  std::vector<T> v(n);
  std::ifstream f(path.c_str(), std::ios::binary);
  if (!f) throw std::runtime_error("cannot open " + path);
  f.read((char *)&v[0], (std::streamsize)(n * sizeof(T)));
  if (!f) throw std::runtime_error("short file " + path);
  return v;
}

template <class T>
static void write_bin(const std::string &path, const std::vector<T> &v) {
  std::ofstream f(path.c_str(), std::ios::binary);
  if (!v.empty()) f.write((const char *)&v[0], (std::streamsize)(v.size() * sizeof(T)));
  if (!f) throw std::runtime_error("cannot write " + path);
}

static double now_s() {
  struct timeval tv;
  gettimeofday(&tv, 0);
  return tv.tv_sec + 1e-6 * tv.tv_usec;
}

// ---------------------------------------------------------------- set-up (main.cc:131-245, one grid)

static void setup(const std::string &deck) {
  Rank = 0;
  np = 1;
  input.setFile(deck + ".in");
  read_inputs();
  const int ngrid = input.section("grid", 0).count;
  if (ngrid != 1) throw std::runtime_error("the driver handles one grid");
  equations.resize(ngrid);
  turbulent.resize(ngrid);
  for (int gid = 0; gid < ngrid; ++gid) {
    if (input.section("grid", gid).get_string("equations") == "navierstokes") equations[gid] = NS;
    else throw std::runtime_error("only navierstokes grids are on this path");
    turbulent[gid] = input.section("grid", gid).subsection("turbulence").is_found;
  }
  grid.resize(ngrid);
  ns.resize(grid.size());
  rans.resize(grid.size());
  hc.resize(grid.size());
  bc.resize(grid.size());
  interface.resize(grid.size());
  for (int gid = 0; gid < (int)grid.size(); ++gid) {
    grid[gid].dimension = input.section("grid", gid).get_int("dimension");
    grid[gid].gid = gid;
    grid[gid].read(input.section("grid", gid).get_string("file"), input.section("grid", gid).get_string("format"));
    grid[gid].raw.type = CELL;
    if (input.section("grid", gid).subsection("transform", 0).count > 0)
      throw std::runtime_error("grid transforms are not used by these cases");
    grid[gid].setup();
    set_bcs(gid);
    define_unset_bc_fields(gid);
    set_lengthScales(gid);
    face_interpolation_weights(gid);
    node_interpolation_weights(gid);
    gradient_maps(gid);
  }
  const int ps_step_max = input.section("pseudotime").get_int("numberofsteps");
  for (int gid = 0; gid < (int)grid.size(); ++gid) {
    ns[gid].gid = gid;
    ns[gid].initialize(ps_step_max);
    if (turbulent[gid]) {
      rans[gid].gid = gid;
      rans[gid].initialize(ps_step_max);
    }
  }
  for (int gid = 0; gid < (int)grid.size(); ++gid) check_bc_fields(gid);
  set_time_step_options();
  set_pseudo_time_step_options();
  loads.resize(grid.size());
  for (int gid = 0; gid < (int)grid.size(); ++gid) {
    Subsection &wo = input.section("grid", gid).subsection("writeoutput");
    loads[gid].moment_center = wo.get_Vec3D("momentcenter");
    loads[gid].frequency = wo.get_int("loadfrequency");
    std::vector<std::string> temp = wo.get_stringList("includebcs");
    loads[gid].force.resize(temp.size());
    loads[gid].moment.resize(temp.size());
    for (size_t i = 0; i < temp.size(); ++i) {
      loads[gid].include_bcs.push_back(atoi(temp[i].c_str()) - 1);
      loads[gid].force[i] = 0.;
      loads[gid].moment[i] = 0.;
    }
  }
}

// ---------------------------------------------------------------- state and residual

static void set_state(const std::vector<double> &W) {
  NavierStokes &N = ns[0];
  const int nc = grid[0].cellCount;
  for (int c = 0; c < nc; ++c) {
    N.p.cell(c) = W[5 * c];
    N.V.cell(c) = Vec3D(W[5 * c + 1], W[5 * c + 2], W[5 * c + 3]);
    N.T.cell(c) = W[5 * c + 4];
    N.rho.cell(c) = N.material.rho(N.p.cell(c), N.T.cell(c));
  }
}

static void set_turbulence(const std::vector<double> &K) {
  RANS &T = rans[0];
  const int nc = grid[0].cellCount;
  for (int c = 0; c < nc; ++c) {
    T.k.cell(c) = K[2 * c];
    T.omega.cell(c) = K[2 * c + 1];
  }
}

// One residual: the reference's order within NavierStokes::solve (ns.cc:104-118)
// with the ghost update first, as after update_variables.
static void residual(bool turb) {
  NavierStokes &N = ns[0];
  N.mpi_update_ghost_primitives();
  N.update_boundaries();
  if (turb) {
    rans[0].mpi_update_ghost_primitives();
    rans[0].update_boundaries();
    rans[0].update_eddy_viscosity();
  }
  N.calc_cell_grads();
  N.mpi_update_ghost_gradients();
  N.calc_limiter();
  VecSet(N.rhs, 0.);
  N.timeStep = 1;
  N.assemble_linear_system();
  if (turb) {
    RANS &T = rans[0];
    T.calc_cell_grads();
    T.mpi_update_ghost_gradients();
    VecSet(T.rhs, 0.);
    T.timeStep = 1;
    T.terms();
  }
}

static void cmd_mesh(const std::string &out) {
  Grid &g = grid[0];
  std::vector<int> fp(g.faceCount), fn(g.faceCount), fb(g.faceCount), fnodes(4 * g.faceCount, -1);
  std::vector<double> fnorm(3 * g.faceCount), farea(g.faceCount), fcen(3 * g.faceCount), favg(2 * g.faceCount);
  for (int f = 0; f < g.faceCount; ++f) {
    fp[f] = g.face[f].parent;
    fn[f] = g.face[f].neighbor;
    fb[f] = g.face[f].bc;
    for (size_t k = 0; k < g.face[f].nodes.size() && k < 4; ++k) fnodes[4 * f + k] = g.face[f].nodes[k];
    for (int k = 0; k < 3; ++k) {
      fnorm[3 * f + k] = g.face[f].normal[k];
      fcen[3 * f + k] = g.face[f].centroid[k];
    }
    farea[f] = g.face[f].area;
    std::map<int, double> &avg = g.face[f].average;
    favg[2 * f] = avg.count(g.face[f].parent) ? avg[g.face[f].parent] : 0.;
    favg[2 * f + 1] = avg.count(g.face[f].neighbor) ? avg[g.face[f].neighbor] : 0.;
  }
  std::vector<int> cfi(1, 0), cf, ni(1, 0), nb, gi(1, 0), gk;
  std::vector<double> gw;
  for (int c = 0; c < g.cellCount; ++c) {
    for (size_t k = 0; k < g.cell[c].faces.size(); ++k) cf.push_back(g.cell[c].faces[k]);
    for (size_t k = 0; k < g.cell[c].neighborCells.size(); ++k) nb.push_back(g.cell[c].neighborCells[k]);
    for (std::map<int, Vec3D>::iterator it = g.cell[c].gradMap.begin(); it != g.cell[c].gradMap.end(); ++it) {
      gk.push_back(it->first);
      for (int k = 0; k < 3; ++k) gw.push_back(it->second[k]);
    }
    cfi.push_back((int)cf.size());
    ni.push_back((int)nb.size());
    gi.push_back((int)gk.size());
  }
  const size_t nt = g.cell.size();
  std::vector<double> cc(3 * nt), cv(nt), cls(nt), cwd(nt);
  for (size_t c = 0; c < nt; ++c) {
    for (int k = 0; k < 3; ++k) cc[3 * c + k] = g.cell[c].centroid[k];
    cv[c] = g.cell[c].volume;
    cls[c] = g.cell[c].lengthScale;
    cwd[c] = g.cell[c].closest_wall_distance;
  }
  write_bin(out + "/face_parent.i32", fp);
  write_bin(out + "/face_neighbor.i32", fn);
  write_bin(out + "/face_bc.i32", fb);
  write_bin(out + "/face_nodes.i32", fnodes);
  write_bin(out + "/cell_face_index.i32", cfi);
  write_bin(out + "/cell_faces.i32", cf);
  write_bin(out + "/nbr_index.i32", ni);
  write_bin(out + "/nbrs.i32", nb);
  write_bin(out + "/grad_index.i32", gi);
  write_bin(out + "/grad_keys.i32", gk);
  write_bin(out + "/grad_weights.f64", gw);
  write_bin(out + "/face_normal.f64", fnorm);
  write_bin(out + "/face_area.f64", farea);
  write_bin(out + "/face_centroid.f64", fcen);
  write_bin(out + "/face_avg.f64", favg);
  write_bin(out + "/cell_centroid.f64", cc);
  write_bin(out + "/cell_volume.f64", cv);
  write_bin(out + "/cell_length.f64", cls);
  write_bin(out + "/cell_wall_distance.f64", cwd);
  std::vector<double> lref(1, g.lengthScale);
  write_bin(out + "/length_scale.f64", lref);
}

static void cmd_residual(const std::string &wpath, const std::string &out, const std::string &kpath) {
  Grid &g = grid[0];
  NavierStokes &N = ns[0];
  const int nc = g.cellCount;
  const bool turb = !kpath.empty();
  if (turb && !turbulent[0]) throw std::runtime_error("a k-omega state needs a deck with a turbulence section");
  set_state(read_bin<double>(wpath, 5 * (size_t)nc));
  if (turb) set_turbulence(read_bin<double>(kpath, 2 * (size_t)nc));
  residual(turb);
  std::vector<double> R(5 * (size_t)nc);
  for (size_t i = 0; i < R.size(); ++i) R[i] = N.rhs->v[i];
  std::vector<double> mdot(g.faceCount), wl(g.faceCount);
  for (int f = 0; f < g.faceCount; ++f) {
    mdot[f] = N.mdot.face(f);
    wl[f] = N.weightL.face(f);
  }
  const size_t nt = g.cell.size();
  std::vector<double> grads(15 * nt), lim(5 * (size_t)nc), ghost(5 * (nt - nc));
  for (size_t c = 0; c < nt; ++c) {
    Vec3D *gs[5] = {&N.gradp.cell(c), &N.gradu.cell(c), &N.gradv.cell(c), &N.gradw.cell(c), &N.gradT.cell(c)};
    for (int v = 0; v < 5; ++v)
      for (int k = 0; k < 3; ++k) grads[15 * c + 3 * v + k] = (*gs[v])[k];
  }
  for (int c = 0; c < nc; ++c)
    for (int v = 0; v < 5; ++v) lim[5 * c + v] = N.limiter[v].cell(c);
  for (size_t c = nc; c < nt; ++c) {
    const size_t k = c - nc;
    ghost[5 * k] = N.p.cell(c);
    ghost[5 * k + 1] = N.V.cell(c)[0];
    ghost[5 * k + 2] = N.V.cell(c)[1];
    ghost[5 * k + 3] = N.V.cell(c)[2];
    ghost[5 * k + 4] = N.T.cell(c);
  }
  write_bin(out + "/R.f64", R);
  write_bin(out + "/mdot.f64", mdot);
  write_bin(out + "/weightL.f64", wl);
  write_bin(out + "/grads.f64", grads);
  write_bin(out + "/limiter.f64", lim);
  write_bin(out + "/ghost.f64", ghost);
  if (turb) {
    RANS &T = rans[0];
    std::vector<double> RK(2 * (size_t)nc), mut(nt);
    for (size_t i = 0; i < RK.size(); ++i) RK[i] = T.rhs->v[i];
    for (size_t c = 0; c < nt; ++c) mut[c] = T.mu_t.cell(c);
    write_bin(out + "/RK.f64", RK);
    write_bin(out + "/mu_t.f64", mut);
  }
}

static void cmd_timeterms(const std::string &wpath, const std::string &dtpath, const std::string &out) {
  Grid &g = grid[0];
  NavierStokes &N = ns[0];
  const int nc = g.cellCount;
  set_state(read_bin<double>(wpath, 5 * (size_t)nc));
  std::vector<double> d = read_bin<double>(dtpath, (size_t)nc);
  for (int c = 0; c < nc; ++c) dt[0].cell(c) = d[c];
  MatZeroEntries(N.impOP);
  fcfd_ref_mat_capture = 1;
  fcfd_ref_mat_cap_lo = 0;
  fcfd_ref_mat_cap_hi = 5 * nc;
  N.ps_step = 1;
  N.time_terms();
  fcfd_ref_mat_capture = 0;
  std::vector<double> blocks(25 * (size_t)nc, 0.);
  for (std::map<std::pair<int, int>, double>::iterator it = N.impOP->entries.begin(); it != N.impOP->entries.end(); ++it) {
    const int r = it->first.first, c = it->first.second;
    if (r / 5 != c / 5) throw std::runtime_error("time_terms wrote an off-diagonal block");
    blocks[25 * (size_t)(r / 5) + 5 * (r % 5) + (c % 5)] = it->second;
  }
  MatZeroEntries(N.impOP);
  write_bin(out + "/blocks.f64", blocks);
}

// Diagonal 5x5 blocks of the reference's implicit operator for state W and
// time steps dt: the first-order finite-difference face Jacobians that
// assemble_linear_system adds (get_jacobians, ns_assemble_linear_system.cc:
// 142-190) plus time_terms' P V / dt; off-diagonal blocks are dropped.
static void cmd_diagblocks(const std::string &wpath, const std::string &dtpath, const std::string &out) {
  Grid &g = grid[0];
  NavierStokes &N = ns[0];
  const int nc = g.cellCount;
  set_state(read_bin<double>(wpath, 5 * (size_t)nc));
  std::vector<double> d = read_bin<double>(dtpath, (size_t)nc);
  for (int c = 0; c < nc; ++c) dt[0].cell(c) = d[c];
  fcfd_ref_mat_capture = 1;
  fcfd_ref_mat_cap_lo = 0;
  fcfd_ref_mat_cap_hi = 5 * nc;
  residual(false);
  N.ps_step = 1;
  N.time_terms();
  fcfd_ref_mat_capture = 0;
  std::vector<double> blocks(25 * (size_t)nc, 0.);
  for (std::map<std::pair<int, int>, double>::iterator it = N.impOP->entries.begin(); it != N.impOP->entries.end(); ++it) {
    const int r = it->first.first, c = it->first.second;
    if (r / 5 != c / 5) continue;
    blocks[25 * (size_t)(r / 5) + 5 * (r % 5) + (c % 5)] = it->second;
  }
  MatZeroEntries(N.impOP);
  write_bin(out + "/blocks.f64", blocks);
}

static void cmd_dt(const std::string &wpath, const std::string &out) {
  const int nc = grid[0].cellCount;
  set_state(read_bin<double>(wpath, 5 * (size_t)nc));
  double time = 0., max_cfl = 0.;
  update_time_step(1, time, max_cfl, 0);
  std::vector<double> d(nc + 2);
  for (int c = 0; c < nc; ++c) d[c] = dt[0].cell(c);
  d[nc] = time;
  d[nc + 1] = max_cfl;
  write_bin(out + "/dt.f64", d);
}

// `evals` timed residual evaluations after `warmup` untimed ones, the state
// reloaded before each (as update_variables would have changed it).
static std::string cmd_bench(const std::string &wpath, int evals, int warmup, const std::string &kpath) {
  const int nc = grid[0].cellCount;
  const bool turb = !kpath.empty();
  const std::vector<double> W = read_bin<double>(wpath, 5 * (size_t)nc);
  std::vector<double> K;
  if (turb) K = read_bin<double>(kpath, 2 * (size_t)nc);
  for (int i = 0; i < warmup; ++i) {
    set_state(W);
    if (turb) set_turbulence(K);
    residual(turb);
  }
  const double t0 = now_s();
  for (int i = 0; i < evals; ++i) {
    set_state(W);
    if (turb) set_turbulence(K);
    residual(turb);
  }
  const double t1 = now_s();
  std::ostringstream s;
  s.precision(17);
  s << "\"evaluations\": " << evals << ", \"seconds\": " << (t1 - t0);
  return s.str();
}

int main(int argc, char **argv) {
  if (argc < 4) {
    std::fprintf(stderr, "usage: %s <case_dir> <deck_basename> mesh|residual|timeterms|dt|bench [args]\n", argv[0]);
    return 2;
  }
  const std::string dir = argv[1], deck = argv[2], cmd = argv[3];
  std::vector<std::string> a;
  for (int i = 4; i < argc; ++i) a.push_back(argv[i]);
  if (chdir(dir.c_str()) != 0) {
    std::fprintf(stderr, "cannot enter %s\n", dir.c_str());
    return 2;
  }
  // The reference's progress messages are not part of any result.
  std::ofstream devnull("/dev/null");
  std::streambuf *saved = std::cout.rdbuf();
  if (!getenv("FCFD_REF_VERBOSE")) std::cout.rdbuf(devnull.rdbuf());
  std::string extra;
  try {
    const double t0 = now_s();
    setup(deck);
    const double t_setup = now_s() - t0;
    std::ostringstream s;
    s.precision(17);
    if (cmd == "mesh" && a.size() == 1) cmd_mesh(a[0]);
    else if (cmd == "residual" && (a.size() == 2 || a.size() == 3)) cmd_residual(a[0], a[1], a.size() == 3 ? a[2] : "");
    else if (cmd == "timeterms" && a.size() == 3) cmd_timeterms(a[0], a[1], a[2]);
    else if (cmd == "dt" && a.size() == 2) cmd_dt(a[0], a[1]);
    else if (cmd == "diagblocks" && a.size() == 3) cmd_diagblocks(a[0], a[1], a[2]);
    else if (cmd == "bench" && (a.size() == 3 || a.size() == 4))
      extra = cmd_bench(a[0], atoi(a[1].c_str()), atoi(a[2].c_str()), a.size() == 4 ? a[3] : "");
    else throw std::runtime_error("unknown command or wrong arguments: " + cmd);
    Grid &g = grid[0];
    long long st = 0, cf = 0;
    for (int c = 0; c < g.cellCount; ++c) {
      st += (long long)g.cell[c].gradMap.size();
      cf += (long long)g.cell[c].faces.size();
    }
    s << "{\"nc\": " << g.cellCount << ", \"nf\": " << g.faceCount << ", \"nghost\": " << (g.cell.size() - g.cellCount)
      << ", \"ntot\": " << g.cell.size() << ", \"nnodes\": " << g.nodeCount << ", \"n_grad_entries\": " << st
      << ", \"n_cell_faces\": " << cf << ", \"setup_seconds\": " << t_setup << ", \"bc\": [";
    for (size_t b = 0; b < bc[0].size(); ++b)
      s << (b ? ", " : "") << "[" << bc[0][b].type << ", " << bc[0][b].kind << ", " << bc[0][b].specified << ", "
        << bc[0][b].thermalType << "]";
    s << "]";
    if (!extra.empty()) s << ", " << extra;
    s << "}";
    std::cout.rdbuf(saved);
    std::cout << "FCFD_REF_RESULT " << s.str() << std::endl;
  } catch (const std::exception &e) {
    std::cout.rdbuf(saved);
    std::fprintf(stderr, "freecfd_ref: %s\n", e.what());
    return 1;
  }
  return 0;
}
