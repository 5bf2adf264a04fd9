// Host-side records shared by the deck reader, the mesh builder and the CUDA
// context.  All arrays are structure-of-arrays, indexed in the reference's
// cell / face order (ghost cells after the interior cells).
#pragma once
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/fcfd.h"

namespace fcfd {

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

void set_last_error(const std::string &m);

// Boundary-condition codes (src/bc.h:28-52)
enum BcType { BC_SYMMETRY = 1, BC_WALL = 2, BC_INLET = 3, BC_OUTLET = 4 };
enum BcKind { K_NONE = -1, K_NO_REVERSE = 1, K_DAMP_REVERSE = 2, K_VELOCITY = 3, K_MDOT = 4, K_SLIP = 5,
              K_STAGNATION = 6, K_FORCE_SUPERSONIC = 7 };
enum BcThermal { TH_FIXED_T = 1, TH_FIXED_Q = 2, TH_ADIABATIC = 3 };
enum BcSpec { SP_RHO = 1, SP_P = 2, SP_T = 3, SP_STATE = 4 };
// Options (src/navier_stokes/ns.h:38-52)
enum Limiter { LIM_NONE = -1, LIM_VK = 1, LIM_BJ = 2, LIM_MINMOD = 3 };
enum Order { ORDER_FIRST = 1, ORDER_SECOND = 2 };
enum Flux { FLUX_ROE = 1, FLUX_VAN_LEER = 2, FLUX_AUSM_PLUS_UP = 3, FLUX_SD_SLAU = 4, FLUX_SW = 5 };
enum GradMethod { GM_CURVILINEAR = 1, GM_LSQR = 2, GM_GREENGAUSS = 3 };
enum Interp { IP_WTLI = 0, IP_IDW = 1, IP_SIMPLE = 2 };

struct BcRegion {
  int type = 0, kind = K_NONE, specified = -1, thermal = -1;
  // region selection (set_bcs.cc:50-69)
  bool box = false;
  double corner1[3] = {0, 0, 0}, corner2[3] = {0, 0, 0};
  std::string pick = "override";
  int pick_from = 0;
  // fixed values (ns_set_bcs.cc)
  bool p_fixed = false, T_fixed = false, rho_fixed = false, V_fixed = false, qdot_fixed = false, mdot_fixed = false;
  double p = 0, T = 0, rho = 0, qdot = 0, mdot = 0, p_total = 0, T_total = 0;
  double V[3] = {0, 0, 0};
  double total_area = 0;  // filled by the mesh builder
  // RANS (rans_set_bcs.cc): inlet turbulence intensity / eddy-viscosity ratio
  double turb_intensity = 1e-4, turb_ratio = 0.1;
};

struct Material {
  double Mw = 28.97, R = 0, gamma = 1.4, Pref = 0, Tref = 0;
  bool sutherland = false, prandtl = false;
  double mu = 0, lambda = 0, sut_mu_ref = 0, sut_T_ref = 0, sut_S = 0, Pr = 0.7;
  double Cp() const { return gamma * R / (gamma - 1.); }
};

// Time marching options (read_inputs.cc:152-176, set_time_step_options
// time_step.cc:25-67): step type, CFL ramp, schedule file, pseudo-time steps.
enum { TS_NONE = 0, TS_FIXED = 1, TS_CFL_MAX = 2, TS_CFL_LOCAL = 3 };
struct TimeMarching {
  int type = TS_NONE;
  double stepsize = 1., cfl_max = 1000., cfl_local = 1000.;
  bool ramp = false;
  double ramp_initial = 1., ramp_growth = 1.2;
  int n_steps = 0, update_freq = 1000000;
  std::string schedule_file;  // empty: none
  int ps_steps = 1;           // pseudotime -> numberofsteps (dual time stepping when > 1)
};
// Faces of a face-based grid (the FACE raw type of grid_reader_tec.cc): node
// lists (0-based global node ids, CSR) and left / right cells (-1: none), in
// file order.
struct FaceInput {
  int n_faces = 0;
  const int32_t *index = nullptr, *nodes = nullptr, *left = nullptr, *right = nullptr;
};

// Parses the timemarching / pseudotime sections of a deck file (also used to
// re-read them every `updatefrequency` steps, update_time_step_options).
TimeMarching read_time_marching(const std::string &path);

}  // namespace fcfd

struct fcfd_case {
  int dimension = 3;
  int flux = fcfd::FLUX_AUSM_PLUS_UP, limiter = fcfd::LIM_VK, order = fcfd::ORDER_SECOND;
  double limiter_threshold = 0, Minf = 1;
  double wdiss = 0.3, bl_height = 0;  // Steger-Warming wall dissipation (ns.cc:76-77)
  int hex_method = fcfd::GM_CURVILINEAR, prism_method = fcfd::GM_CURVILINEAR, other_method = fcfd::GM_LSQR;
  int interp = fcfd::IP_WTLI, stencil_size = 2;
  fcfd::Material mat;
  std::vector<fcfd::BcRegion> bc;
  double cfl_max = 1000, cfl_local = 1000;
  bool has_cfl_max = false, has_cfl_local = false;
  // driver options: time marching, output frequencies (main.cc:227-249), the
  // linear-solver tolerances of navierstokes (ns.cc:37-39), the deck's path
  fcfd::TimeMarching tm;
  int restart_freq = 1000000, load_freq = 1000000;
  double moment_center[3] = {0., 0., 0.};
  std::vector<int> load_bcs;  // writeoutput -> includebcs, 0-based
  double lin_rtol = 1e-6, lin_abstol = 1e-12;
  int lin_maxits = 10;
  std::string deck_path;
  // turbulence (rans.cc:48-70)
  bool turbulent = false;
  std::string turb_model;
  double k_low = 1e-10, k_high = 1e8, omega_low = 1e-2, visc_ratio_limit = 1e8, Pr_t = 0.9;
  // uniform initial state of IC_1 (the NS face values RANS::set_bcs reads)
  double ic_p = 0, ic_T = 0, ic_rho = 0, ic_V[3] = {0, 0, 0};
  bool ic_has_p = false, ic_has_T = false, ic_has_rho = false;
};

struct fcfd_mesh {
  int32_t nc = 0, nf = 0, nb = 0, nnode = 0, dimension = 3;
  // faces (reference order)
  std::vector<int32_t> f_parent, f_neighbor, f_bc, f_nodes;  // f_nodes: [nf][4], -1 pad
  std::vector<uint8_t> f_nn;                                 // node count
  std::vector<double> f_normal, f_area, f_centroid, f_w;     // f_w: [nf][2] averaging weights (parent, neighbor)
  std::vector<double> f_t1, f_t2;                            // tangents (face_geom_update)
  std::vector<uint8_t> f_symmetry;
  // cells: interior [0,nc), ghosts [nc, nc+nb)
  std::vector<double> c_centroid, c_volume, c_length, c_wall;
  std::vector<double> f_wall, f_diss;                         // face wall distance / dissipation factor (Steger-Warming only)
  std::vector<int32_t> c_bc;                                 // ghost -> bc index (-1 interior)
  std::vector<int32_t> cf_index, cf_list;                    // interior cell -> faces (ascending)
  std::vector<int32_t> nbr_index, nbr_list;                  // interior cell -> neighborCells
  // LSQ data (lsqr_grad_map): stencil keys in ascending order (self included)
  std::vector<int32_t> st_index, st_keys;
  std::vector<double> st_cof;                                // [nc][7]: C00 C01 C02 C11 C12 C22 det
  std::vector<double> st_self;                               // [nc][3]: self weight
  std::vector<double> st_recip;                              // [nc]: 1/det where the reciprocal division is exact, else 0
  std::vector<double> st_mirror;                             // [nc][3]: sum of the symmetry-mirror weights
  std::vector<uint8_t> has_lsq;                              // 1 if gradMap non-empty
  // gradient maps as weights per stencil entry ([E][3], key order), built
  // when some cell takes the curvilinear map (curvilinear_grad_map.cc)
  bool grad_weights = false;
  std::vector<double> st_w;
  std::vector<int32_t> color_index, color_cells;             // face-neighbour colouring
  std::vector<double> nodes;                                 // [nnode][3]
  double length_scale = 0, total_volume = 0;
  std::vector<double> bc_total_area;
};
