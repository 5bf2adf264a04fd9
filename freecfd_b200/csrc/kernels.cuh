// Device kernels of the finite-volume residual, templated on the scalar type S.
//
// Data layout (all reference-order, structure-of-arrays):
//   W[5][nt]        primitive state p,u,v,w,T of interior cells [0,nc) and
//                   boundary ghosts [nc,nt)
//   G[15][nc]       cell gradients (p,u,v,w,T) x (x,y,z)
//   L[5][nc]        limiters
//   D[5][nf]        per-face F_diffusive - F_convective
//   R               residual, gathered per cell in ascending face order
// Kernel chain per residual: ghost+minmax -> grad+limiter -> (outlet density)
// -> face flux -> gather.  The chain mirrors update_boundaries,
// calc_cell_grads, calc_limiter and the face loop of assemble_linear_system.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

namespace fcfd {

// ------------------------------------------------------------------ scalar ops
// Parity-critical sums (LSQ gradient, limiter tests) are evaluated with
// explicitly rounded operations so no multiply-add is contracted and the
// result is the same double the reference computes.
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double div_rn(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float div_rn(float a, float b) { return __fdiv_rn(a, b); }


// ------------------------------------------------------------------ dual numbers
// Forward tangent arithmetic: value v and directional derivative d.  Branches
// and comparisons use the value, so a kernel instantiated on Dual computes the
// residual's directional derivative along the seeded direction exactly
// (hand-differentiated forward mode of the same code, no finite difference).
template <class T>
struct Dual {
  T v, d;
  __host__ __device__ Dual() : v(0), d(0) {}
  __host__ __device__ Dual(double x) : v(T(x)), d(0) {}
  __host__ __device__ Dual(T x, T y) : v(x), d(y) {}
};
template <class T> __host__ __device__ __forceinline__ Dual<T> operator+(const Dual<T> &a, const Dual<T> &b) { return Dual<T>(a.v + b.v, a.d + b.d); }
template <class T> __host__ __device__ __forceinline__ Dual<T> operator-(const Dual<T> &a, const Dual<T> &b) { return Dual<T>(a.v - b.v, a.d - b.d); }
template <class T> __host__ __device__ __forceinline__ Dual<T> operator-(const Dual<T> &a) { return Dual<T>(-a.v, -a.d); }
template <class T> __host__ __device__ __forceinline__ Dual<T> operator*(const Dual<T> &a, const Dual<T> &b) { return Dual<T>(a.v * b.v, a.d * b.v + a.v * b.d); }
template <class T> __host__ __device__ __forceinline__ Dual<T> operator/(const Dual<T> &a, const Dual<T> &b) {
  const T q = a.v / b.v;
  return Dual<T>(q, (a.d - q * b.d) / b.v);
}
template <class T> __host__ __device__ __forceinline__ Dual<T> operator+(const Dual<T> &a, double b) { return Dual<T>(a.v + T(b), a.d); }
template <class T> __host__ __device__ __forceinline__ Dual<T> operator+(double a, const Dual<T> &b) { return Dual<T>(T(a) + b.v, b.d); }
template <class T> __host__ __device__ __forceinline__ Dual<T> operator-(const Dual<T> &a, double b) { return Dual<T>(a.v - T(b), a.d); }
template <class T> __host__ __device__ __forceinline__ Dual<T> operator-(double a, const Dual<T> &b) { return Dual<T>(T(a) - b.v, -b.d); }
template <class T> __host__ __device__ __forceinline__ Dual<T> operator*(const Dual<T> &a, double b) { return Dual<T>(a.v * T(b), a.d * T(b)); }
template <class T> __host__ __device__ __forceinline__ Dual<T> operator*(double a, const Dual<T> &b) { return Dual<T>(T(a) * b.v, T(a) * b.d); }
template <class T> __host__ __device__ __forceinline__ Dual<T> operator/(const Dual<T> &a, double b) { return Dual<T>(a.v / T(b), a.d / T(b)); }
template <class T> __host__ __device__ __forceinline__ Dual<T> operator/(double a, const Dual<T> &b) {
  const T q = T(a) / b.v;
  return Dual<T>(q, -q * b.d / b.v);
}
#define FCFD_DUAL_CMP(op)                                                                                                  \
  template <class T> __host__ __device__ __forceinline__ bool operator op(const Dual<T> &a, const Dual<T> &b) { return a.v op b.v; } \
  template <class T> __host__ __device__ __forceinline__ bool operator op(const Dual<T> &a, double b) { return a.v op T(b); }        \
  template <class T> __host__ __device__ __forceinline__ bool operator op(double a, const Dual<T> &b) { return T(a) op b.v; }
FCFD_DUAL_CMP(<)
FCFD_DUAL_CMP(>)
FCFD_DUAL_CMP(<=)
FCFD_DUAL_CMP(>=)
FCFD_DUAL_CMP(==)
FCFD_DUAL_CMP(!=)
#undef FCFD_DUAL_CMP
template <class T> __host__ __device__ __forceinline__ Dual<T> sqrt(const Dual<T> &a) {
  const T s = sqrt(a.v);
  return Dual<T>(s, a.d / (T(2) * s));
}
template <class T> __host__ __device__ __forceinline__ Dual<T> fabs(const Dual<T> &a) { return a.v < T(0) ? -a : a; }
template <class T> __host__ __device__ __forceinline__ Dual<T> pow(const Dual<T> &a, double e) {
  const T p = pow(a.v, T(e));
  return Dual<T>(p, a.d == T(0) ? T(0) : T(e) * p / a.v * a.d);
}
template <class T> __host__ __device__ __forceinline__ Dual<T> tanh(const Dual<T> &a) {
  const T t = tanh(a.v);
  return Dual<T>(t, (T(1) - t * t) * a.d);
}
using ::fabs;
using ::pow;
using ::sqrt;
using ::tanh;
__device__ __forceinline__ Dual<double> mul_rn(Dual<double> a, Dual<double> b) { return Dual<double>(__dmul_rn(a.v, b.v), a.d * b.v + a.v * b.d); }
__device__ __forceinline__ Dual<double> add_rn(Dual<double> a, Dual<double> b) { return Dual<double>(__dadd_rn(a.v, b.v), a.d + b.d); }
__device__ __forceinline__ Dual<double> sub_rn(Dual<double> a, Dual<double> b) { return Dual<double>(__dsub_rn(a.v, b.v), a.d - b.d); }
__device__ __forceinline__ Dual<double> div_rn(Dual<double> a, Dual<double> b) {
  const double q = __ddiv_rn(a.v, b.v);
  return Dual<double>(q, (a.d - q * b.d) / b.v);
}
__device__ __forceinline__ Dual<float> mul_rn(Dual<float> a, Dual<float> b) { return Dual<float>(__fmul_rn(a.v, b.v), a.d * b.v + a.v * b.d); }
__device__ __forceinline__ Dual<float> add_rn(Dual<float> a, Dual<float> b) { return Dual<float>(__fadd_rn(a.v, b.v), a.d + b.d); }
__device__ __forceinline__ Dual<float> sub_rn(Dual<float> a, Dual<float> b) { return Dual<float>(__fsub_rn(a.v, b.v), a.d - b.d); }
__device__ __forceinline__ Dual<float> div_rn(Dual<float> a, Dual<float> b) {
  const float q = __fdiv_rn(a.v, b.v);
  return Dual<float>(q, (a.d - q * b.d) / b.v);
}
// ------------------------------------------------------------------ FP32 scalar
// The scalar of the FP32 face pass of the mixed-precision residual: float
// storage and float arithmetic, with every double operand (case constants,
// geometry) rounded to float first -- the arithmetic Dual<float> gives its
// value part, without the tangent.  A plain `float` would not do: the
// kernels' double constants would promote each expression back to FP64.
struct F32 {
  float v;
  __host__ __device__ F32() : v(0.f) {}
  __host__ __device__ F32(double x) : v(float(x)) {}
  __host__ __device__ static F32 of(float x) {
    F32 r;
    r.v = x;
    return r;
  }
};
__host__ __device__ __forceinline__ F32 operator+(F32 a, F32 b) { return F32::of(a.v + b.v); }
__host__ __device__ __forceinline__ F32 operator-(F32 a, F32 b) { return F32::of(a.v - b.v); }
__host__ __device__ __forceinline__ F32 operator*(F32 a, F32 b) { return F32::of(a.v * b.v); }
__host__ __device__ __forceinline__ F32 operator/(F32 a, F32 b) { return F32::of(a.v / b.v); }
__host__ __device__ __forceinline__ F32 operator-(F32 a) { return F32::of(-a.v); }
__host__ __device__ __forceinline__ F32 operator+(F32 a, double b) { return F32::of(a.v + float(b)); }
__host__ __device__ __forceinline__ F32 operator+(double a, F32 b) { return F32::of(float(a) + b.v); }
__host__ __device__ __forceinline__ F32 operator-(F32 a, double b) { return F32::of(a.v - float(b)); }
__host__ __device__ __forceinline__ F32 operator-(double a, F32 b) { return F32::of(float(a) - b.v); }
__host__ __device__ __forceinline__ F32 operator*(F32 a, double b) { return F32::of(a.v * float(b)); }
__host__ __device__ __forceinline__ F32 operator*(double a, F32 b) { return F32::of(float(a) * b.v); }
__host__ __device__ __forceinline__ F32 operator/(F32 a, double b) { return F32::of(a.v / float(b)); }
__host__ __device__ __forceinline__ F32 operator/(double a, F32 b) { return F32::of(float(a) / b.v); }
#define FCFD_F32_CMP(op)                                                                                   \
  __host__ __device__ __forceinline__ bool operator op(F32 a, F32 b) { return a.v op b.v; }                \
  __host__ __device__ __forceinline__ bool operator op(F32 a, double b) { return a.v op float(b); }        \
  __host__ __device__ __forceinline__ bool operator op(double a, F32 b) { return float(a) op b.v; }
FCFD_F32_CMP(<)
FCFD_F32_CMP(>)
FCFD_F32_CMP(<=)
FCFD_F32_CMP(>=)
FCFD_F32_CMP(==)
FCFD_F32_CMP(!=)
#undef FCFD_F32_CMP
__host__ __device__ __forceinline__ F32 sqrt(F32 a) { return F32::of(sqrtf(a.v)); }
__host__ __device__ __forceinline__ F32 fabs(F32 a) { return F32::of(fabsf(a.v)); }
__host__ __device__ __forceinline__ F32 pow(F32 a, double e) { return F32::of(powf(a.v, float(e))); }
__host__ __device__ __forceinline__ F32 tanh(F32 a) { return F32::of(tanhf(a.v)); }
__device__ __forceinline__ F32 mul_rn(F32 a, F32 b) { return F32::of(__fmul_rn(a.v, b.v)); }
__device__ __forceinline__ F32 add_rn(F32 a, F32 b) { return F32::of(__fadd_rn(a.v, b.v)); }
__device__ __forceinline__ F32 sub_rn(F32 a, F32 b) { return F32::of(__fsub_rn(a.v, b.v)); }
__device__ __forceinline__ F32 div_rn(F32 a, F32 b) { return F32::of(__fdiv_rn(a.v, b.v)); }
__host__ __device__ __forceinline__ float val(F32 x) { return x.v; }
__host__ __device__ __forceinline__ double tan_of(F32) { return 0.; }

__host__ __device__ __forceinline__ double val(double x) { return x; }
__host__ __device__ __forceinline__ float val(float x) { return x; }
template <class T> __host__ __device__ __forceinline__ T val(const Dual<T> &x) { return x.v; }
__host__ __device__ __forceinline__ double tan_of(double) { return 0.; }
template <class S> struct Mk;
template <> struct Mk<double> { __host__ __device__ static double of(double v, double) { return v; } };
template <> struct Mk<F32> { __host__ __device__ static F32 of(double v, double) { return F32(v); } };
template <class T> struct Mk<Dual<T>> { __host__ __device__ static Dual<T> of(double v, double d) { return Dual<T>(T(v), T(d)); } };
template <class T> __host__ __device__ __forceinline__ T tan_of(const Dual<T> &x) { return x.d; }

// std::max / std::min semantics: max(a,b) = (a<b)?b:a, min(a,b) = (b<a)?b:a
// Runs the statement with the compile-time flux selector FX of face_D bound
// to the case's convective flux (4 SD-SLAU, 5 Steger-Warming, else 0).
#define FCFD_BY_FLUX(flux, ...)                       \
  do {                                                \
    if ((flux) == 4) {                                \
      constexpr int FX = 4;                           \
      __VA_ARGS__;                                    \
    } else if ((flux) == 5) {                         \
      constexpr int FX = 5;                           \
      __VA_ARGS__;                                    \
    } else {                                          \
      constexpr int FX = 0;                           \
      __VA_ARGS__;                                    \
    }                                                 \
  } while (0)

// Programmatic dependent launch.  A kernel launched with the programmatic
// stream-serialization attribute may be scheduled while its predecessor in
// the stream is still running: pdl_wait() blocks until every prerequisite grid
// has completed and its writes are visible (a no-op for an ordinary launch),
// so each kernel of the residual chain calls it before touching any array;
// pdl_trigger() lets the successor be scheduled as this grid's last blocks
// run, so its launch overlaps this kernel's tail.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

template <class S> __host__ __device__ __forceinline__ S smax(const S &a, const S &b) { return (a < b) ? b : a; }
template <class S> __host__ __device__ __forceinline__ S smin(const S &a, const S &b) { return (b < a) ? b : a; }

// ------------------------------------------------------------------ case data
struct DevBC {
  int type, kind, specified, thermal;
  double p, T, rho, qdot, mdot_per_area, p_total, T_total;
  double V[3];
  // Variable fixedonBC flags the RANS terms read (T face value, k / omega /
  // eddy viscosity BC values of rans_set_bcs.cc)
  int T_fixed, kw_fixed, mut_fixed, pad_;
  double k_bc, omega_bc, mut_bc;
  int p_fixed, V_fixed;  // p / V fixed on the BC (their Green-Gauss face values)
};
constexpr int kMaxBC = 16;
struct DevCase {
  double gamma, R, Pref, Tref, Minf, K, Lref, Cp;
  double mu, lambda, sut_mu_ref, sut_T_ref, sut_S, Pr;
  double Pr_t;
  double wdiss, bl_height;  // Steger-Warming wall dissipation and boundary-layer height
  int sutherland, prandtl, flux, limiter, order, viscous, nbc, frozen_limiter;
  int fast_grad;
  int pair_grad;  // every cell has a gradient stencil: the two-threads-per-cell gradient may run
  int tile_grad;  // the shared-memory tile gradient kernel runs (DevMesh tiles built)
  int fold_grad;  // the fused gradient sums the folded stencils (DevMesh fold_* built)
  DevBC bc[kMaxBC];
};

struct DevMesh {
  int nc, nf, nb, nt;
  const int *f_parent, *f_neighbor, *f_bc;
  const double *f_n, *f_area, *f_x, *f_w;  // f_n/f_x: [3][nf] SoA, f_w: [2][nf]
  const double *c_x;                       // [3][nt]
  const double *c_len;                     // [nc]
  const int *cf_index, *cf_list;           // cf_list: face id, ~face id when the cell is the neighbour
  const int *st_index, *st_keys;
  const double *st_cof;                    // [7][nc]
  const double *st_self;                   // [3][nc]
  const double *st_recip;                  // [nc] 1/det where the reciprocal division is exact, else 0
  const double *c_vol;                     // [nc] cell volumes (Green-Gauss gradients)
  const double *st_mirror;                 // [3][nc] summed symmetry-mirror weights
  const double *st_w = nullptr;            // [E][3] stored map weights (curvilinear cases), else null
  // tiles of the shared-memory gradient kernel (null: not built): the staged
  // cells of tile t are tile_cells[tile_off[t], tile_off[t+1]); st_local and
  // cf_local give a stencil entry's / face entry's cell as a slot in its
  // cell's tile, self_local the cell's own slot
  const int *tile_off = nullptr, *tile_cells = nullptr, *st_local = nullptr, *cf_local = nullptr,
            *self_local = nullptr;
  int tile_slots_max = 0;
  // least-squares stencils with the symmetry ghosts of z-normal planes folded
  // into their parents' entries (null: not built): per cell the entries
  // [fold_index[c], fold_index[c+1]), entry j naming cell fold_key[j] with
  // the weighted offsets fold_e[6j..6j+2] = w d of the cell itself and
  // fold_e[6j+3..6j+5] = sum of w d over its mirror ghosts in the stencil
  const int *fold_index = nullptr, *fold_key = nullptr;
  const double *fold_e = nullptr;
  const int *bface;                        // boundary faces in ghost order [nb]
  const int *outlet_faces;                 // outlet boundary faces [n_outlet]
  const double *f_wall, *f_diss;           // [nf] wall distance, dissipation factor (Steger-Warming only)
  int n_outlet;
  // Faces of the viscous or partitioned main face-flux launch, thread i
  // taking face_list[i]: the whole mesh grouped by kind (interior faces, then
  // each BC region's, each group in face order) so that a warp's faces take
  // the same branch, or one rank's faces of a domain decomposition, grouped
  // the same way.
  const int *face_list = nullptr;
  int n_face_list = 0;
  // Partitioned evaluation (one rank of a domain decomposition; null lists =
  // the whole mesh): cells whose gradient and limiter are formed, indices
  // into outlet_faces, ghost indices to update, and the owned cells
  // [own_lo, own_hi) (extrema and gather).
  const int *part_cells = nullptr, *part_outlet = nullptr, *part_ghosts = nullptr;
  int n_part_cells = 0, n_part_outlet = 0, n_part_ghosts = 0;
  int own_lo = 0, own_hi = 0;
};
// thread counts of the ghost and gather kernels (partition-aware)
__host__ __device__ inline int n_ghost_threads(const DevMesh &m) { return m.part_ghosts ? m.n_part_ghosts : m.nb; }
__host__ __device__ inline int n_owned(const DevMesh &m) { return m.part_cells ? m.own_hi - m.own_lo : m.nc; }

enum { T_SYM = 1, T_WALL = 2, T_INLET = 3, T_OUTLET = 4 };
enum { KN_NONE = -1, KN_NO_REVERSE = 1, KN_DAMP_REVERSE = 2, KN_VELOCITY = 3, KN_MDOT = 4, KN_SLIP = 5, KN_STAGNATION = 6,
       KN_FORCE_SUPERSONIC = 7 };
enum { SP_RHO_ = 1, SP_P_ = 2, SP_T_ = 3, SP_STATE_ = 4 };
enum { TH_FIXED_T_ = 1, TH_FIXED_Q_ = 2 };
enum { ERR_SUPERSONIC_INLET = 1, ERR_BAD_BC = 2 };

// material (material/material.cc:108-153)
template <class S> __host__ __device__ __forceinline__ S eos_rho(const DevCase &c, S p, S T) { return (p + c.Pref) / (c.R * (T + c.Tref)); }
template <class S> __host__ __device__ __forceinline__ S eos_p(const DevCase &c, S rho, S T) { return rho * c.R * (T + c.Tref) - c.Pref; }
template <class S> __host__ __device__ __forceinline__ S eos_T(const DevCase &c, S p, S rho) { return (p + c.Pref) / (c.R * rho) - c.Tref; }
template <class S> __host__ __device__ __forceinline__ S sound(const DevCase &c, S p, S T) { return sqrt(c.gamma * (p + c.Pref) / eos_rho(c, p, T)); }
template <class S> __device__ __forceinline__ S viscosity(const DevCase &c, S T) {
  if (!c.sutherland) return S(c.mu);
  // Sutherland (material.cc:126-131); t^1.5 as t * sqrt(t) (the reference's
  // pow(t, 1.5) to rounding, at a fraction of pow's instructions)
  const S t = (T + c.Tref) / c.sut_T_ref;
  return c.sut_mu_ref * (t * sqrt(t)) * (c.sut_T_ref + c.sut_S) / (T + c.Tref + c.sut_S);
}
template <class S> __device__ __forceinline__ S therm_cond(const DevCase &c, S T) {
  if (!c.prandtl) return S(c.lambda);
  return c.Cp * viscosity(c, T) / c.Pr;
}

// face-local state (NS_Cell_State without the rotated frame)
template <class S>
struct FState {
  S p, T, rho, a, H, Vn;
  S V[3];
  S pc, Tc;
  S Vc[3];
};

template <class S>
__host__ __device__ __forceinline__ void finish(const DevCase &c, FState<S> &s, const double n[3]) {
  s.a = sound(c, s.p, s.T);
  s.H = s.a * s.a / (c.gamma - 1.) + 0.5 * (s.V[0] * s.V[0] + s.V[1] * s.V[1] + s.V[2] * s.V[2]);
  s.Vn = s.V[0] * n[0] + s.V[1] * n[1] + s.V[2] * n[2];
}

// finish() for a state whose rho was just set to eos_rho(p, T): the sound
// speed reuses that density instead of recomputing it (the same doubles as
// finish(); the low-Mach energy flux cancels so strongly that even a
// one-rounding change of a or H shows in the residual).
template <class S>
__host__ __device__ __forceinline__ void finish_eos(const DevCase &c, FState<S> &s, const double n[3]) {
  s.a = sqrt(c.gamma * (s.p + c.Pref) / s.rho);
  s.H = s.a * s.a / (c.gamma - 1.) + 0.5 * (s.V[0] * s.V[0] + s.V[1] * s.V[1] + s.V[2] * s.V[2]);
  s.Vn = s.V[0] * n[0] + s.V[1] * n[1] + s.V[2] * n[2];
}

// Boundary right state (ns_apply_bcs.cc:25-258).  Returns false when the
// branch leaves R.rho untouched (outlet with everything extrapolated), in which
// case the caller supplies the density the reference's state cache held.
template <class S>
__device__ bool apply_bc(const DevCase &c, const DevBC &b, const FState<S> &L, FState<S> &R, const double n[3], int *err) {
  const double g = c.gamma;
  const S uNL = L.V[0] * n[0] + L.V[1] * n[1] + L.V[2] * n[2];
  bool rho_set = true;
  if (b.type == T_INLET) {
    if (b.kind == KN_VELOCITY) {
      R.V[0] = S(b.V[0]); R.V[1] = S(b.V[1]); R.V[2] = S(b.V[2]);
      S uNR = R.V[0] * n[0] + R.V[1] * n[1] + R.V[2] * n[2];
      R.a = L.a + 0.5 * (uNL - uNR) * (g - 1.);
      S MachL = -uNL / L.a;
      if (MachL >= 1. && b.specified != SP_STATE_ && err) atomicOr(err, ERR_SUPERSONIC_INLET);
      if (b.specified == SP_STATE_) { R.p = S(b.p); R.T = S(b.T); R.rho = S(b.rho); }
      else if (b.specified == SP_P_) { R.p = S(b.p); R.rho = g * (R.p + c.Pref) / (R.a * R.a); R.T = eos_T(c, R.p, R.rho); }
      else if (b.specified == SP_T_) {
        R.T = S(b.T);
        R.rho = L.rho * pow((L.T + c.Tref) / (R.T + c.Tref), 1. / (1. - g));
        R.p = eos_p(c, R.rho, R.T);
      } else if (b.specified == SP_RHO_) { R.rho = S(b.rho); R.p = R.a * R.a * R.rho / g - c.Pref; R.T = eos_T(c, R.p, R.rho); }
      else if (err) atomicOr(err, ERR_BAD_BC);
      R.pc = R.p; R.Tc = R.T; R.Vc[0] = R.V[0]; R.Vc[1] = R.V[1]; R.Vc[2] = R.V[2];
    } else if (b.kind == KN_MDOT) {
      const double mdotNR = -1. * b.mdot_per_area;
      if (b.specified == SP_STATE_) { R.p = S(b.p); R.T = S(b.T); R.rho = S(b.rho); }
      else if (b.specified == SP_P_) { R.p = S(b.p); R.T = L.T; R.rho = eos_rho(c, R.p, R.T); }
      else if (b.specified == SP_T_) { R.T = S(b.T); R.p = L.p; R.rho = eos_rho(c, R.p, R.T); }
      else if (b.specified == SP_RHO_) {
        R.rho = S(b.rho);
        R.a = 0.5 * (g - 1.) * (uNL + 2. * L.a / (g - 1.) - mdotNR / R.rho);
        R.p = R.a * R.a * R.rho / g - c.Pref;
        R.T = eos_T(c, R.p, R.rho);
      } else if (err) atomicOr(err, ERR_BAD_BC);
      S s = mdotNR / R.rho;
      R.V[0] = s * n[0]; R.V[1] = s * n[1]; R.V[2] = s * n[2];
      R.pc = R.p; R.Tc = R.T; R.Vc[0] = R.V[0]; R.Vc[1] = R.V[1]; R.Vc[2] = R.V[2];
    } else if (b.kind == KN_STAGNATION) {
      if (uNL > 0.) { R.V[0] = -1. * L.Vc[0]; R.V[1] = -1. * L.Vc[1]; R.V[2] = -1. * L.Vc[2]; }
      else { R.V[0] = L.Vc[0]; R.V[1] = L.Vc[1]; R.V[2] = L.Vc[2]; }
      S v2 = R.V[0] * R.V[0] + R.V[1] * R.V[1] + R.V[2] * R.V[2];
      R.T = b.T_total - 0.5 * (g - 1.) / (g * c.R) * v2;
      R.p = (b.p_total + c.Pref) / (1. + 0.5 * v2 / (c.R * (R.T + c.Tref))) - c.Pref;
      R.rho = eos_rho(c, R.p, R.T);
      R.pc = R.p; R.Tc = R.T; R.Vc[0] = R.V[0]; R.Vc[1] = R.V[1]; R.Vc[2] = R.V[2];
    } else {
      rho_set = false;  // inlet without V/mdot/p_total: the reference applies nothing
    }
  } else if (b.type == T_OUTLET) {
    S MachL = uNL / L.a;
    bool supersonic = (MachL > 1.);
    const double ig = 1. / g;
    if (b.specified == SP_P_ && !supersonic) {
      R.p = S(b.p); R.pc = R.p;
      R.rho = L.rho * pow((R.p + c.Pref), ig) / pow((L.p + c.Pref), ig);
      R.a = sqrt(g * (R.p + c.Pref) / R.rho);
      R.T = eos_T(c, R.p, R.rho);
      R.V[0] = L.V[0]; R.V[1] = L.V[1]; R.V[2] = L.V[2];
    } else if (b.specified == SP_T_ && !supersonic) {
      R.T = S(b.T); R.Tc = R.T;
      R.a = sqrt(g * c.R * (R.T + c.Tref));
      R.rho = pow(g * (L.p + c.Pref) / (R.a * R.a * pow(L.rho, g)), 1. - g);
      R.p = eos_p(c, R.rho, R.T);
      R.V[0] = L.V[0]; R.V[1] = L.V[1]; R.V[2] = L.V[2];
    } else if (b.specified == SP_RHO_ && !supersonic) {
      R.rho = S(b.rho);
      R.p = (L.p + c.Pref) * pow(R.rho / L.rho, g) - c.Pref;
      R.T = eos_T(c, R.p, R.rho);
      R.a = sqrt(g * (R.p + c.Pref) / R.rho);
      R.V[0] = L.V[0]; R.V[1] = L.V[1]; R.V[2] = L.V[2];
    } else {
      R.p = L.p; R.T = L.T; R.V[0] = L.V[0]; R.V[1] = L.V[1]; R.V[2] = L.V[2];
      rho_set = false;
    }
    if (MachL < 0.) {
      if (b.kind == KN_DAMP_REVERSE) {
        R.p = R.p - 0.5 * L.rho * uNL * uNL;
        R.rho = L.rho * pow((R.p + c.Pref), ig) / pow((L.p + c.Pref), ig);
        R.a = sqrt(g * (R.p + c.Pref) / R.rho);
        R.T = eos_T(c, R.p, R.rho);
        rho_set = true;
      }
      if (b.kind == KN_NO_REVERSE) { R.V[0] = -1. * L.V[0]; R.V[1] = -1. * L.V[1]; R.V[2] = -1. * L.V[2]; }
    }
    if (MachL < 1. && b.kind == KN_FORCE_SUPERSONIC) {
      S d = L.a - uNL;
      R.p = R.p - 0.5 * L.rho * (d * d);
      R.p = smin(S(1.e-8), R.p + c.Pref) - c.Pref;
      R.rho = L.rho * pow((R.p + c.Pref), ig) / pow((L.p + c.Pref), ig);
      R.a = sqrt(g * (R.p + c.Pref) / R.rho);
      R.T = eos_T(c, R.p, R.rho);
      rho_set = true;
    }
  } else if (b.type == T_WALL) {
    if (b.thermal == TH_FIXED_T_) {
      R.T = S(b.T); R.Tc = R.T;
      R.p = L.p;
      R.rho = eos_rho(c, R.p, R.T);
    } else {
      R.p = L.p; R.rho = L.rho; R.T = L.T; R.Tc = L.Tc;
    }
    if (b.kind == KN_SLIP) {
      S s = 2. * uNL;
      R.V[0] = L.V[0] - s * n[0]; R.V[1] = L.V[1] - s * n[1]; R.V[2] = L.V[2] - s * n[2];
      S sc = 2. * (L.Vc[0] * n[0] + L.Vc[1] * n[1] + L.Vc[2] * n[2]);
      R.Vc[0] = L.Vc[0] - sc * n[0]; R.Vc[1] = L.Vc[1] - sc * n[1]; R.Vc[2] = L.Vc[2] - sc * n[2];
    } else {
      R.V[0] = -1. * L.V[0]; R.V[1] = -1. * L.V[1]; R.V[2] = -1. * L.V[2];
      R.Vc[0] = -1. * L.Vc[0]; R.Vc[1] = -1. * L.Vc[1]; R.Vc[2] = -1. * L.Vc[2];
    }
    R.pc = L.pc;
  } else if (b.type == T_SYM) {
    R.p = L.p;
    S s = 2. * uNL;
    R.V[0] = L.V[0] - s * n[0]; R.V[1] = L.V[1] - s * n[1]; R.V[2] = L.V[2] - s * n[2];
    R.T = L.T;
    R.rho = L.rho;
    R.pc = L.pc;
    R.Tc = L.Tc;
    S sc = 2. * (L.Vc[0] * n[0] + L.Vc[1] * n[1] + L.Vc[2] * n[2]);
    R.Vc[0] = L.Vc[0] - sc * n[0]; R.Vc[1] = L.Vc[1] - sc * n[1]; R.Vc[2] = L.Vc[2] - sc * n[2];
  } else {
    rho_set = false;
  }
  return rho_set;
}

// Centre state of cell k as a face state (zero gradients).
template <class S>
__device__ __forceinline__ void centre_state(const DevCase &c, const S *W, int nt, int k, FState<S> &s, const double n[3]) {
  s.p = W[k]; s.V[0] = W[nt + k]; s.V[1] = W[2 * nt + k]; s.V[2] = W[3 * nt + k]; s.T = W[4 * nt + k];
  s.pc = s.p; s.Tc = s.T; s.Vc[0] = s.V[0]; s.Vc[1] = s.V[1]; s.Vc[2] = s.V[2];
  s.rho = eos_rho(c, s.p, s.T);
  finish(c, s, n);
}

// Reconstructed state of cell k at face point xf (left_state_update,
// ns_assemble_linear_system.cc:269-294).
// SA: the element type of W, G, Lm (S itself, or double under the FP32 face
// pass of the mixed-precision residual, which loads FP64 arrays).
template <class S, class SA = S>
__device__ __forceinline__ void recon_state(const DevCase &c, const DevMesh &m, const SA *W, const SA *G, const SA *Lm, int k,
                                            const double xf[3], FState<S> &s, const double n[3]) {
  const int nt = m.nt, nc = m.nc;
  const double d0 = xf[0] - m.c_x[k], d1 = xf[1] - m.c_x[nt + k], d2 = xf[2] - m.c_x[2 * nt + k];
  S q[5];
#pragma unroll
  for (int v = 0; v < 5; ++v) {
    S dot = d0 * G[(3 * v) * nc + k] + d1 * G[(3 * v + 1) * nc + k] + d2 * G[(3 * v + 2) * nc + k];
    q[v] = W[v * nt + k] + Lm[v * nc + k] * dot;
  }
  s.pc = W[k]; s.Vc[0] = W[nt + k]; s.Vc[1] = W[2 * nt + k]; s.Vc[2] = W[3 * nt + k]; s.Tc = W[4 * nt + k];
  s.p = q[0]; s.V[0] = q[1]; s.V[1] = q[2]; s.V[2] = q[3]; s.T = q[4];
  s.rho = eos_rho(c, s.p, s.T);
  finish_eos(c, s, n);
}

// ------------------------------------------------------------------ kernels

// Green-Gauss gradient of cell c (Variable::cell_gradient's fallback for an
// empty gradient map, variable.h:204-213): sum over the cell's faces in
// ascending order of the face value x (n A / V), negated on the neighbour
// side; the face value is the BC value where the variable is fixed on the BC,
// else the face average w_p phi_p + w_n phi_n.  Rounded operations in the
// reference's order.
template <class S>
__device__ void green_gauss(const DevCase &cs, const DevMesh &m, const S *__restrict__ W, int c, S g[15]) {
  const int nt = m.nt, nf = m.nf;
  const double vol = m.c_vol[c];
#pragma unroll
  for (int i = 0; i < 15; ++i) g[i] = S(0.);
  for (int j = m.cf_index[c]; j < m.cf_index[c + 1]; ++j) {
    const int e = m.cf_list[j];
    const int f = e >= 0 ? e : ~e;
    const double A = m.f_area[f];
    double av[3];
    for (int i = 0; i < 3; ++i) {
      av[i] = div_rn(mul_rn(m.f_n[i * nf + f], A), vol);
      if (e < 0) av[i] = mul_rn(av[i], -1.);
    }
    const int b = m.f_bc[f], pa = m.f_parent[f], nb = m.f_neighbor[f];
    const double w0 = m.f_w[f], w1 = m.f_w[nf + f];
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      S fv;
      bool fixed = false;
      if (b >= 0) {
        const DevBC &bc = cs.bc[b];
        if (v == 0 && bc.p_fixed) { fv = S(bc.p); fixed = true; }
        else if (v == 4 && bc.T_fixed) { fv = S(bc.T); fixed = true; }
        else if (v >= 1 && v <= 3 && bc.V_fixed) { fv = S(bc.V[v - 1]); fixed = true; }
      }
      if (!fixed) fv = add_rn(add_rn(S(0.), mul_rn(S(w0), W[v * nt + pa])), mul_rn(S(w1), W[v * nt + nb]));
#pragma unroll
      for (int i = 0; i < 3; ++i) g[3 * v + i] = add_rn(g[3 * v + i], mul_rn(fv, S(av[i])));
    }
  }
}

// AoS [nc][5] -> SoA W[5][nt]
template <class S>
__global__ void k_aos_to_soa(const S *__restrict__ in, S *__restrict__ W, int nc, int nt) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
#pragma unroll
  for (int v = 0; v < 5; ++v) W[v * nt + c] = in[5 * c + v];
}

__device__ __forceinline__ unsigned long long okey(double x) {
  unsigned long long b = __double_as_longlong(x);
  return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double okey_inv(unsigned long long k) {
  unsigned long long b = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
  return __longlong_as_double(b);
}

// Ghost update (reconstructed NavierStokes::update_boundaries, first order)
// over boundary faces, plus the global extrema that find_min_max
// (ns.cc:400-435) needs: slots 0..7 = max p, min p, max u, min u, max v,
// min v, max p over cells < nc-1, min p over cells < nc-1 (ordered keys).
template <class S>
__global__ void k_ghost_minmax(DevCase cs, DevMesh m, S *__restrict__ W, unsigned long long *__restrict__ ext, int *err) {
  pdl_wait();
  pdl_trigger();
  const int nt = m.nt;
  const int nbl = n_ghost_threads(m);
  const int ghost_blocks = (nbl + blockDim.x - 1) / blockDim.x;
  if ((int)blockIdx.x < ghost_blocks) {
    int tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= nbl) return;
    if (m.part_ghosts) tid = m.part_ghosts[tid];
    const int f = m.bface[tid];
    const int pa = m.f_parent[f];
    const int b = m.f_bc[f];
    const double n[3] = {m.f_n[f], m.f_n[m.nf + f], m.f_n[2 * m.nf + f]};
    FState<S> L, R;
    centre_state(cs, W, nt, pa, L, n);
    R.rho = S(0.);
    apply_bc(cs, cs.bc[b], L, R, n, err);
    const int g = m.nc + tid;
    W[g] = R.p; W[nt + g] = R.V[0]; W[2 * nt + g] = R.V[1]; W[3 * nt + g] = R.V[2]; W[4 * nt + g] = R.T;
    return;
  }
  if (!ext) return;
  // The remaining blocks reduce the interior extrema: grid-stride, warp
  // shuffles, a shared-memory block reduction and one atomic per block/slot.
  const int eb = blockIdx.x - ghost_blocks, neb = gridDim.x - ghost_blocks;
  double mx[4] = {-INFINITY, -INFINITY, -INFINITY, -INFINITY}, mn[4] = {INFINITY, INFINITY, INFINITY, INFINITY};
  // over the owned cells of a partition (global ids, so the quirk slots keep
  // their meaning), else over all interior cells
  const int c0 = m.part_cells ? m.own_lo : 0, c1 = m.part_cells ? m.own_hi : m.nc;
  for (int c = c0 + eb * blockDim.x + threadIdx.x; c < c1; c += neb * blockDim.x) {
    const double p = val(W[c]), u = val(W[nt + c]), v = val(W[2 * nt + c]);
    mx[0] = fmax(mx[0], p); mn[0] = fmin(mn[0], p);
    mx[1] = fmax(mx[1], u); mn[1] = fmin(mn[1], u);
    mx[2] = fmax(mx[2], v); mn[2] = fmin(mn[2], v);
    if (c < m.nc - 1) { mx[3] = fmax(mx[3], p); mn[3] = fmin(mn[3], p); }
  }
  __shared__ double smx[4][32], smn[4][32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    for (int o = 16; o > 0; o >>= 1) {
      mx[i] = fmax(mx[i], __shfl_xor_sync(0xffffffffu, mx[i], o));
      mn[i] = fmin(mn[i], __shfl_xor_sync(0xffffffffu, mn[i], o));
    }
    if (lane == 0) { smx[i][wid] = mx[i]; smn[i][wid] = mn[i]; }
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    const int i = threadIdx.x;
    double a = -INFINITY, b = INFINITY;
    for (int k = 0; k < nw; ++k) { a = fmax(a, smx[i][k]); b = fmin(b, smn[i][k]); }
    const int slot_max[4] = {0, 2, 4, 6}, slot_min[4] = {1, 3, 5, 7};
    if (a != -INFINITY) atomicMax(&ext[slot_max[i]], okey(a));
    if (b != INFINITY) atomicMin(&ext[slot_min[i]], okey(b));
  }
}

// First cell attaining each extreme (tangent runs): slots as in k_ghost_minmax.
template <class S>
__global__ void k_argext(DevMesh m, const S *__restrict__ W, const unsigned long long *__restrict__ ext, int *__restrict__ argx) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= m.nc) return;
  const int nt = m.nt;
  const double p = val(W[c]), u = val(W[nt + c]), v = val(W[2 * nt + c]);
  if (p == okey_inv(ext[0])) atomicMin(&argx[0], c);
  if (p == okey_inv(ext[1])) atomicMin(&argx[1], c);
  if (u == okey_inv(ext[2])) atomicMin(&argx[2], c);
  if (u == okey_inv(ext[3])) atomicMin(&argx[3], c);
  if (v == okey_inv(ext[4])) atomicMin(&argx[4], c);
  if (v == okey_inv(ext[5])) atomicMin(&argx[5], c);
  if (c < m.nc - 1) {
    if (p == okey_inv(ext[6])) atomicMin(&argx[6], c);
    if (p == okey_inv(ext[7])) atomicMin(&argx[7], c);
  }
}

// Combine a value array and a tangent array (AoS [nc][5]) into SoA duals.
template <class T>
__global__ void k_seed_dual(const double *__restrict__ w, const double *__restrict__ dw, Dual<T> *__restrict__ W, int nc, int nt) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
#pragma unroll
  for (int v = 0; v < 5; ++v) W[v * nt + c] = Dual<T>(T(w[5 * c + v]), T(dw[5 * c + v]));
}

// Split a dual SoA result into value and tangent AoS arrays.
template <class T>
__global__ void k_split_dual(const Dual<T> *__restrict__ R, double *__restrict__ r, double *__restrict__ dr, int nc) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
#pragma unroll
  for (int v = 0; v < 5; ++v) {
    const Dual<T> x = R[v * nc + c];
    if (r) r[5 * c + v] = double(x.v);
    dr[5 * c + v] = double(x.d);
  }
}

// Cell data of the gradient + limiter body: states W and centroids c_x of
// the cells a stencil entry or a face neighbour names, from global memory
// (cell ids), or from a tile staged in shared memory (slots).
template <class S>
struct CellsGlobal {
  const S *W;
  const double *cx;
  int nt;
  __device__ __forceinline__ S w(int v, int k) const { return W[v * nt + k]; }
  __device__ __forceinline__ double x(int i, int k) const { return cx[i * nt + k]; }
  // stencil entry j's cell, the cell itself, the other cell of face entry j
  __device__ __forceinline__ int key(const DevMesh &m, int j) const { return m.st_keys[j]; }
  __device__ __forceinline__ int self(int c) const { return c; }
  __device__ __forceinline__ int nbr(const DevMesh &m, int j, int e) const {
    const int f = e >= 0 ? e : ~e;
    return e >= 0 ? m.f_neighbor[f] : m.f_parent[f];
  }
};
struct CellsTile {
  const double *sW, *sX;  // [5][ns], [3][ns] in shared memory
  int ns, self_slot;
  const int *st_local, *cf_local;
  __device__ __forceinline__ double w(int v, int s) const { return sW[v * ns + s]; }
  __device__ __forceinline__ double x(int i, int s) const { return sX[i * ns + s]; }
  __device__ __forceinline__ int key(const DevMesh &, int j) const { return st_local[j]; }
  __device__ __forceinline__ int self(int) const { return self_slot; }
  __device__ __forceinline__ int nbr(const DevMesh &, int j, int) const { return cf_local[j]; }
};

// Fused least-squares sums over the folded stencil entries [j0, j1) of cell
// c: entry j names cell k with E0 = w d of k itself (zero for c) and Eg = the
// sum of w d over k's mirror ghosts across z-normal symmetry planes in c's
// stencil; those ghosts hold (p, u, v, -w, T) of k, so
//   acc_v += (phi_k - phi_c) (E0 + Eg)        for p, u, v, T
//   acc_w += (w_k - w_c) E0 + (-w_k - w_c) Eg
// which is the unfolded sum over all the entries, regrouped.
template <class S>
__device__ __forceinline__ void fold_sum(const DevMesh &m, const S *__restrict__ W, int nt, int c, const S u0[5],
                                         S acc[15], int j0, int j1) {
#pragma unroll 2
  for (int j = j0; j < j1; ++j) {
    const int k = m.fold_key[j];
    const double *E = m.fold_e + 6 * (size_t)j;
    const double a0 = E[0], a1 = E[1], a2 = E[2], b0 = E[3], b1 = E[4], b2 = E[5];
    const double s0 = a0 + b0, s1 = a1 + b1, s2 = a2 + b2;
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      const S phi = W[v * nt + k];
      if (v == 3) {
        const S q0 = phi - u0[3], qg = -1. * phi - u0[3];
        acc[9] = acc[9] + q0 * a0 + qg * b0;
        acc[10] = acc[10] + q0 * a1 + qg * b1;
        acc[11] = acc[11] + q0 * a2 + qg * b2;
      } else {
        const S q = phi - u0[v];
        acc[3 * v] = acc[3 * v] + q * s0;
        acc[3 * v + 1] = acc[3 * v + 1] + q * s1;
        acc[3 * v + 2] = acc[3 * v + 2] + q * s2;
      }
    }
  }
}

// LSQ gradient (bit-exact restatement of Variable::cell_gradient over the
// lsqr_grad_map weights) + limiter of interior cell c, reading the cells it
// needs through the accessor A (W itself is read directly only for the VK
// extrema quirks: cells 0 and nc-1).
template <class S, bool FAST, class A>
__device__ __forceinline__ void grad_limiter_cell(const DevCase &cs, const DevMesh &m, const S *__restrict__ W,
                                                  const unsigned long long *__restrict__ ext,
                                                  const int *__restrict__ argx, int c, const A &cells,
                                                  S *__restrict__ G, S *__restrict__ Lm) {
  const int nc = m.nc, nt = m.nt;
  const int cself = cells.self(c);
  const double xc0 = cells.x(0, cself), xc1 = cells.x(1, cself), xc2 = cells.x(2, cself);
  S g[15];
#pragma unroll
  for (int i = 0; i < 15; ++i) g[i] = S(0.);
  const int j0 = m.st_index[c], j1 = m.st_index[c + 1];
  if (j0 == j1) {
    green_gauss(cs, m, W, c, g);
  } else if (FAST) {
    // Continuous limiters only (VK with K > 0, none, first order): the same
    // weighted least-squares gradient in the compact form
    //   grad = C . sum_k w_k d_k (phi_k - phi_c) / det - mirror * phi_c
    // with fused multiply-adds (equal to the reference's sum up to rounding).
    S u0[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) u0[v] = cells.w(v, cself);
    S acc[15];
#pragma unroll
    for (int i = 0; i < 15; ++i) acc[i] = S(0.);
    if constexpr (std::is_same<A, CellsGlobal<S>>::value) {
      if (cs.fold_grad) {
        // folded stencil: a z-normal symmetry ghost holds its parent's state
        // with w negated, so its term w (phi_g - phi_c) d joins the parent's
        fold_sum(m, cells.W, nt, c, u0, acc, m.fold_index[c], m.fold_index[c + 1]);
      }
    }
#pragma unroll 4
    for (int j = (std::is_same<A, CellsGlobal<S>>::value && cs.fold_grad) ? j1 : j0; j < j1; ++j) {
      const int k = cells.key(m, j);
      if (k == cself) continue;
      const double d0 = cells.x(0, k) - xc0, d1 = cells.x(1, k) - xc1, d2 = cells.x(2, k) - xc2;
      const double w = d0 * d0 + d1 * d1 + d2 * d2;
#pragma unroll
      for (int v = 0; v < 5; ++v) {
        const S a = w * (cells.w(v, k) - u0[v]);
        acc[3 * v] = acc[3 * v] + a * d0;
        acc[3 * v + 1] = acc[3 * v + 1] + a * d1;
        acc[3 * v + 2] = acc[3 * v + 2] + a * d2;
      }
    }
    const double C00 = m.st_cof[c], C01 = m.st_cof[nc + c], C02 = m.st_cof[2 * nc + c];
    const double C11 = m.st_cof[3 * nc + c], C12 = m.st_cof[4 * nc + c], C22 = m.st_cof[5 * nc + c];
    const double id = 1. / m.st_cof[6 * nc + c];
    const double M0 = m.st_mirror[c], M1 = m.st_mirror[nc + c], M2 = m.st_mirror[2 * nc + c];
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      const S s0 = acc[3 * v], s1 = acc[3 * v + 1], s2 = acc[3 * v + 2];
      g[3 * v] = (C00 * s0 + C01 * s1 + C02 * s2) * id - M0 * u0[v];
      g[3 * v + 1] = (C01 * s0 + C11 * s1 + C12 * s2) * id - M1 * u0[v];
      g[3 * v + 2] = (C02 * s0 + C12 * s1 + C22 * s2) * id - M2 * u0[v];
    }
  } else {
    // Bit-exact: every weight rebuilt with the reference's rounded operations.
    // The division by det uses the reciprocal with one fused correction where
    // the mesh builder verified it returns the IEEE quotient for every weight.
    // (Weights precomputed on the host and streamed from HBM measured slower:
    // 200 against 190 us on the prism mesh.)
    if (m.st_w) {
      // stored map weights (curvilinear maps, and the least-squares maps of a
      // mesh that has any): grad += weight * phi in key order
      for (int j = j0; j < j1; ++j) {
        const int k = cells.key(m, j);
        const double wt0 = m.st_w[3 * (size_t)j], wt1 = m.st_w[3 * (size_t)j + 1], wt2 = m.st_w[3 * (size_t)j + 2];
#pragma unroll
        for (int v = 0; v < 5; ++v) {
          const S phi = cells.w(v, k);
          g[3 * v] = add_rn(g[3 * v], mul_rn(S(wt0), phi));
          g[3 * v + 1] = add_rn(g[3 * v + 1], mul_rn(S(wt1), phi));
          g[3 * v + 2] = add_rn(g[3 * v + 2], mul_rn(S(wt2), phi));
        }
      }
    }
    const double C00 = m.st_cof[c], C01 = m.st_cof[nc + c], C02 = m.st_cof[2 * nc + c];
    const double C11 = m.st_cof[3 * nc + c], C12 = m.st_cof[4 * nc + c], C22 = m.st_cof[5 * nc + c];
    const double det = m.st_cof[6 * nc + c];
    const double rc = m.st_recip[c];
    auto qdiv = [&](double x) -> double {
      if (rc != 0.) {
        const double q0 = __dmul_rn(x, rc);
        const double rem = __fma_rn(-q0, det, x);
        return __fma_rn(rem, rc, q0);
      }
      return __ddiv_rn(x, det);
    };
    for (int j = m.st_w ? j1 : j0; j < j1; ++j) {
      const int k = cells.key(m, j);
      double wt0, wt1, wt2;
      if (k == cself) {
        wt0 = m.st_self[c]; wt1 = m.st_self[nc + c]; wt2 = m.st_self[2 * nc + c];
      } else {
        const double d0 = sub_rn(cells.x(0, k), xc0), d1 = sub_rn(cells.x(1, k), xc1), d2 = sub_rn(cells.x(2, k), xc2);
        const double w = add_rn(add_rn(mul_rn(d0, d0), mul_rn(d1, d1)), mul_rn(d2, d2));
        wt0 = qdiv(mul_rn(w, add_rn(add_rn(mul_rn(d0, C00), mul_rn(d1, C01)), mul_rn(d2, C02))));
        wt1 = qdiv(mul_rn(w, add_rn(add_rn(mul_rn(d0, C01), mul_rn(d1, C11)), mul_rn(d2, C12))));
        wt2 = qdiv(mul_rn(w, add_rn(add_rn(mul_rn(d0, C02), mul_rn(d1, C12)), mul_rn(d2, C22))));
      }
#pragma unroll
      for (int v = 0; v < 5; ++v) {
        const S phi = cells.w(v, k);
        g[3 * v] = add_rn(g[3 * v], mul_rn(S(wt0), phi));
        g[3 * v + 1] = add_rn(g[3 * v + 1], mul_rn(S(wt1), phi));
        g[3 * v + 2] = add_rn(g[3 * v + 2], mul_rn(S(wt2), phi));
      }
    }
  }
#pragma unroll
  for (int i = 0; i < 15; ++i) G[i * nc + c] = g[i];

  // ---- limiter (ns_limiters.cc)
  S phi[5];
  const S one = S(cs.order == 1 ? 0. : 1.);
#pragma unroll
  for (int v = 0; v < 5; ++v) phi[v] = one;
  if (cs.order != 1 && cs.limiter > 0) {
    const int f0 = m.cf_index[c], f1 = m.cf_index[c + 1];
    S u0[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) { u0[v] = cells.w(v, cself); phi[v] = S(1.); }
    if (cs.limiter == 3) {
      // minmod (ns_limiters.cc:45-92)
      const double small = 1.e-12;
      for (int j = f0; j < f1; ++j) {
        const int e = m.cf_list[j];
        const int f = e >= 0 ? e : ~e;
        const int nb = cells.nbr(m, j, e);
        const double cf0 = sub_rn(m.f_x[f], xc0), cf1 = sub_rn(m.f_x[m.nf + f], xc1), cf2 = sub_rn(m.f_x[2 * m.nf + f], xc2);
#pragma unroll
        for (int v = 0; v < 5; ++v) {
          S dU = sub_rn(cells.w(v, nb), u0[v]);
          S dUg = add_rn(add_rn(mul_rn(g[3 * v], S(cf0)), mul_rn(g[3 * v + 1], S(cf1))), mul_rn(g[3 * v + 2], S(cf2)));
          S mm;
          if (dU * dUg < 0.) mm = S(0.);
          else if (dU > 0.) mm = smin(dU, dUg);
          else mm = smax(dU, dUg);
          const double sU = (double)((mm > 0.) - (mm < 0.)), sG = (double)((dUg > 0.) - (dUg < 0.));
          S r = div_rn(add_rn(mm, S(sU * small)), add_rn(dUg, S(sG * small)));
          phi[v] = smin(phi[v], r);
        }
      }
    } else {
      // Venkatakrishnan (ns_limiters.cc:161-248) and Barth-Jespersen (94-159)
      S umax[5], umin[5];
#pragma unroll
      for (int v = 0; v < 5; ++v) umax[v] = umin[v] = u0[v];
      for (int j = f0; j < f1; ++j) {
        const int e = m.cf_list[j];
        const int nb = cells.nbr(m, j, e);
#pragma unroll
        for (int v = 0; v < 5; ++v) {
          const S x = cells.w(v, nb);
          umax[v] = smax(umax[v], x);
          umin[v] = smin(umin[v], x);
        }
      }
      S eps2[5] = {S(0.), S(0.), S(0.), S(0.), S(0.)};
      if (cs.limiter == 1) {
        // find_min_max with its index quirks: q[3] uses q[4]'s running value,
        // q[4] tracks p starting from T of cell 0.  std::max keeps the earlier
        // operand on ties, so each extreme belongs to a definite cell; `argx`
        // (tangent runs only) holds the first cell attaining slots 0..7.
        const double pmax = okey_inv(ext[0]), pmin = okey_inv(ext[1]);
        const double T0 = val(W[4 * nt + 0]), wl = val(W[3 * nt + nc - 1]);
        const double tT0 = tan_of(W[4 * nt + 0]), twl = tan_of(W[3 * nt + nc - 1]);
        auto tp = [&](int slot) { return argx ? tan_of(W[argx[slot]]) : 0.; };
        auto tv = [&](int var, int slot) { return argx ? tan_of(W[var * nt + argx[slot]]) : 0.; };
        double qmax[5], qmin[5], tmax[5], tmin[5];
        qmax[0] = pmax; tmax[0] = tp(0); qmin[0] = pmin; tmin[0] = tp(1);
        qmax[1] = okey_inv(ext[2]); tmax[1] = tv(1, 2); qmin[1] = okey_inv(ext[3]); tmin[1] = tv(1, 3);
        qmax[2] = okey_inv(ext[4]); tmax[2] = tv(2, 4); qmin[2] = okey_inv(ext[5]); tmin[2] = tv(2, 5);
        double q4M = T0, t4M = tT0, q4m = T0, t4m = tT0;  // running q[4] before the last cell
        if (nc > 1) {
          const double a = okey_inv(ext[6]), b = okey_inv(ext[7]);
          if (T0 < a) { q4M = a; t4M = tp(6); }
          if (b < T0) { q4m = b; t4m = tp(7); }
        }
        qmax[3] = q4M; tmax[3] = t4M; if (q4M < wl) { qmax[3] = wl; tmax[3] = twl; }
        qmin[3] = q4m; tmin[3] = t4m; if (wl < q4m) { qmin[3] = wl; tmin[3] = twl; }
        qmax[4] = T0; tmax[4] = tT0; if (T0 < pmax) { qmax[4] = pmax; tmax[4] = tp(0); }
        qmin[4] = T0; tmin[4] = tT0; if (pmin < T0) { qmin[4] = pmin; tmin[4] = tp(1); }
#pragma unroll
        for (int v = 0; v < 5; ++v) {
          const S eps = fabs(Mk<S>::of(qmax[v], tmax[v]) - Mk<S>::of(qmin[v], tmin[v])) / cs.Lref;
          const S e = 1.e-6 * cs.K * eps;
          eps2[v] = e * e;
        }
      }
      for (int j = f0; j < f1; ++j) {
        const int e = m.cf_list[j];
        const int f = e >= 0 ? e : ~e;
        const double cf0 = sub_rn(m.f_x[f], xc0), cf1 = sub_rn(m.f_x[m.nf + f], xc1), cf2 = sub_rn(m.f_x[2 * m.nf + f], xc2);
#pragma unroll
        for (int v = 0; v < 5; ++v) {
          S dM = add_rn(add_rn(mul_rn(g[3 * v], S(cf0)), mul_rn(g[3 * v + 1], S(cf1))), mul_rn(g[3 * v + 2], S(cf2)));
          S dP = u0[v];
          if (cs.limiter == 1) {
            if (dM > 0.) dP = sub_rn(umax[v], dP);
            else if (dM < 0.) dP = sub_rn(umin[v], dP);
            const S dP2 = mul_rn(dP, dP), dM2 = mul_rn(dM, dM);
            const S e2 = eps2[v];
            if (dM != 0.) {
              const S num = add_rn(add_rn(dP2, e2), mul_rn(mul_rn(S(2.), dM), dP));
              const S den = add_rn(add_rn(add_rn(dP2, mul_rn(S(2.), dM2)), mul_rn(dM, dP)), e2);
              phi[v] = smin(phi[v], div_rn(num, den));
            }
          } else {
            if (dM > 0.) dP = sub_rn(umax[v], dP);
            else if (dM < 0.) dP = sub_rn(umin[v], dP);
            else { dP = S(1.); dM = S(1.); }
            phi[v] = smin(phi[v], div_rn(dP, dM));
          }
        }
      }
    }
  }
  if (cs.frozen_limiter) {
    // tangent runs for Newton-Krylov: treat the limiter as a constant
#pragma unroll
    for (int v = 0; v < 5; ++v) phi[v] = Mk<S>::of(val(phi[v]), 0.);
  }
#pragma unroll
  for (int v = 0; v < 5; ++v) Lm[v * nc + c] = phi[v];
}

template <class S, bool FAST, bool PART = false>
__global__ void __launch_bounds__(128, (!FAST && std::is_same<S, double>::value) ? 6 : 1) k_grad_limiter(DevCase cs, DevMesh m, const S *__restrict__ W,
                                                      const unsigned long long *__restrict__ ext, const int *__restrict__ argx,
                                                      S *__restrict__ G, S *__restrict__ Lm) {
  pdl_wait();
  pdl_trigger();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  // PART: one rank's gradient cells of a domain decomposition
  int c = i;
  if constexpr (PART) {
    if (i >= m.n_part_cells) return;
    c = m.part_cells[i];
  } else {
    if (i >= m.nc) return;
  }
  const CellsGlobal<S> cells{W, m.c_x, m.nt};
  grad_limiter_cell<S, FAST>(cs, m, W, ext, argx, c, cells, G, Lm);
}

// The same body over tiles of kGradTile consecutive cells, one block per
// tile: the states and centroids of every cell the tile's stencils and faces
// name (the tile's staged set, sorted by cell id, so the loads run along
// ascending addresses) are copied into shared memory once, and the stencil
// and limiter loops read them from there through precomputed slot indices
// (st_local, cf_local, self_local) instead of gathering each from L2 by its
// cell id.  Least-squares meshes without Green-Gauss cells, FP64, whole mesh.
constexpr int kGradTile = 128;
template <bool FAST>
__global__ void __launch_bounds__(kGradTile) k_grad_limiter_tile(DevCase cs, DevMesh m, const double *__restrict__ W,
                                                                 const unsigned long long *__restrict__ ext,
                                                                 double *__restrict__ G, double *__restrict__ Lm) {
  extern __shared__ double tile_smem[];
  pdl_wait();
  pdl_trigger();
  const int t = blockIdx.x, nt = m.nt;
  const int s0 = m.tile_off[t], ns = m.tile_off[t + 1] - s0;
  double *sW = tile_smem, *sX = tile_smem + 5 * ns;
  for (int s = threadIdx.x; s < ns; s += kGradTile) {
    const int k = m.tile_cells[s0 + s];
#pragma unroll
    for (int v = 0; v < 5; ++v) sW[v * ns + s] = W[v * nt + k];
#pragma unroll
    for (int i = 0; i < 3; ++i) sX[i * ns + s] = m.c_x[i * nt + k];
  }
  __syncthreads();
  const int c = t * kGradTile + threadIdx.x;
  if (c >= m.nc) return;
  const CellsTile cells{sW, sX, ns, m.self_local[c], m.st_local, m.cf_local};
  grad_limiter_cell<double, FAST>(cs, m, W, ext, nullptr, c, cells, G, Lm);
}

// LSQ gradient + continuous limiter (VK with K > 0, none, first order), FP64,
// two threads per cell for meshes too small to fill the GPU with one thread
// per cell.  A block is 32 consecutive cells and two warps: warp h takes half
// h of every cell's stencil entries (so each warp reads the j-th entries of 32
// consecutive cells, the coalesced pattern of k_grad_limiter) and half of its
// faces in the limiter's two face loops; partial sums, extremes and limiter
// minima meet in shared memory.  Same operations as k_grad_limiter's FAST path
// except that the stencil sum is formed in two parts.  Cells with an
// empty gradient map (Green-Gauss) are not handled (DevCase::pair_grad).
// PART: one rank's gradient cells of a domain decomposition.
template <bool PART = false>
__global__ void __launch_bounds__(64) k_grad_limiter_pair(DevCase cs, DevMesh m, const double *__restrict__ W,
                                                          const unsigned long long *__restrict__ ext,
                                                          double *__restrict__ G, double *__restrict__ Lm) {
  __shared__ double part[2][15][32];
  pdl_wait();
  pdl_trigger();
  const int lane = threadIdx.x & 31, h = threadIdx.x >> 5;
  const int nc = m.nc, nt = m.nt;
  const int ncell = PART ? m.n_part_cells : nc;
  const int ci = blockIdx.x * 32 + lane;
  const bool act = ci < ncell;
  const int c = act ? (PART ? m.part_cells[ci] : ci) : 0;
  double acc[15];
#pragma unroll
  for (int i = 0; i < 15; ++i) acc[i] = 0.;
  double u0[5] = {0., 0., 0., 0., 0.};
  double xc0 = 0., xc1 = 0., xc2 = 0.;
  if (act) {
    xc0 = m.c_x[c]; xc1 = m.c_x[nt + c]; xc2 = m.c_x[2 * nt + c];
#pragma unroll
    for (int v = 0; v < 5; ++v) u0[v] = W[v * nt + c];
    if (cs.fold_grad) {
      const int f0 = m.fold_index[c], f1 = m.fold_index[c + 1], fm = (f0 + f1) >> 1;
      fold_sum(m, W, nt, c, u0, acc, h == 0 ? f0 : fm, h == 0 ? fm : f1);
    }
    const int j0 = m.st_index[c], j1 = m.st_index[c + 1], mid = (j0 + j1) >> 1;
    const int a = h == 0 ? j0 : mid, b = cs.fold_grad ? a : (h == 0 ? mid : j1);
#pragma unroll 4
    for (int j = a; j < b; ++j) {
      const int k = m.st_keys[j];
      if (k == c) continue;
      const double d0 = m.c_x[k] - xc0, d1 = m.c_x[nt + k] - xc1, d2 = m.c_x[2 * nt + k] - xc2;
      const double w = d0 * d0 + d1 * d1 + d2 * d2;
#pragma unroll
      for (int v = 0; v < 5; ++v) {
        const double q = w * (W[v * nt + k] - u0[v]);
        acc[3 * v] = acc[3 * v] + q * d0;
        acc[3 * v + 1] = acc[3 * v + 1] + q * d1;
        acc[3 * v + 2] = acc[3 * v + 2] + q * d2;
      }
    }
  }
#pragma unroll
  for (int i = 0; i < 15; ++i) part[h][i][lane] = acc[i];
  __syncthreads();
  double g[15];
  {
    const double C00 = m.st_cof[c], C01 = m.st_cof[nc + c], C02 = m.st_cof[2 * nc + c];
    const double C11 = m.st_cof[3 * nc + c], C12 = m.st_cof[4 * nc + c], C22 = m.st_cof[5 * nc + c];
    const double id = 1. / m.st_cof[6 * nc + c];
    const double M0 = m.st_mirror[c], M1 = m.st_mirror[nc + c], M2 = m.st_mirror[2 * nc + c];
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      const double s0 = part[0][3 * v][lane] + part[1][3 * v][lane];
      const double s1 = part[0][3 * v + 1][lane] + part[1][3 * v + 1][lane];
      const double s2 = part[0][3 * v + 2][lane] + part[1][3 * v + 2][lane];
      g[3 * v] = (C00 * s0 + C01 * s1 + C02 * s2) * id - M0 * u0[v];
      g[3 * v + 1] = (C01 * s0 + C11 * s1 + C12 * s2) * id - M1 * u0[v];
      g[3 * v + 2] = (C02 * s0 + C12 * s1 + C22 * s2) * id - M2 * u0[v];
    }
  }
  // warp 0 writes the gradients of p, u, v; warp 1 those of w, T
  if (act) {
#pragma unroll
    for (int i = 0; i < 15; ++i)
      if ((h == 0) == (i < 9)) G[i * nc + c] = g[i];
  }
  double phi[5];
#pragma unroll
  for (int v = 0; v < 5; ++v) phi[v] = cs.order == 1 ? 0. : 1.;
  if (cs.order != 1 && cs.limiter == 1) {
    // the cell's faces are split between the warps as its stencil was: the
    // neighbour extremes and the per-face limiter values are each reduced over
    // both halves through shared memory (max, min: independent of the order)
    __shared__ double ext_s[2][10][32];
    __shared__ double phi_s[2][5][32];
    const int f0 = act ? m.cf_index[c] : 0, f1 = act ? m.cf_index[c + 1] : 0, fm = (f0 + f1) >> 1;
    const int fa = h == 0 ? f0 : fm, fb = h == 0 ? fm : f1;
    double umax[5], umin[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) umax[v] = umin[v] = u0[v];
#pragma unroll 2
    for (int j = fa; j < fb; ++j) {
      const int e = m.cf_list[j];
      const int f = e >= 0 ? e : ~e;
      const int nb = e >= 0 ? m.f_neighbor[f] : m.f_parent[f];
#pragma unroll
      for (int v = 0; v < 5; ++v) {
        const double x = W[v * nt + nb];
        umax[v] = smax(umax[v], x);
        umin[v] = smin(umin[v], x);
      }
    }
#pragma unroll
    for (int v = 0; v < 5; ++v) { ext_s[h][v][lane] = umax[v]; ext_s[h][5 + v][lane] = umin[v]; }
    // find_min_max with its index quirks (see k_grad_limiter)
    double eps2[5];
    {
      const double pmax = okey_inv(ext[0]), pmin = okey_inv(ext[1]);
      const double T0 = W[4 * nt + 0], wl = W[3 * nt + nc - 1];
      double qmax[5], qmin[5];
      qmax[0] = pmax; qmin[0] = pmin;
      qmax[1] = okey_inv(ext[2]); qmin[1] = okey_inv(ext[3]);
      qmax[2] = okey_inv(ext[4]); qmin[2] = okey_inv(ext[5]);
      double q4M = T0, q4m = T0;
      if (nc > 1) {
        const double a = okey_inv(ext[6]), b = okey_inv(ext[7]);
        if (T0 < a) q4M = a;
        if (b < T0) q4m = b;
      }
      qmax[3] = q4M; if (q4M < wl) qmax[3] = wl;
      qmin[3] = q4m; if (wl < q4m) qmin[3] = wl;
      qmax[4] = T0; if (T0 < pmax) qmax[4] = pmax;
      qmin[4] = T0; if (pmin < T0) qmin[4] = pmin;
#pragma unroll
      for (int v = 0; v < 5; ++v) {
        const double eps = fabs(qmax[v] - qmin[v]) / cs.Lref;
        const double e = 1.e-6 * cs.K * eps;
        eps2[v] = e * e;
      }
    }
    __syncthreads();
#pragma unroll
    for (int v = 0; v < 5; ++v) {
      umax[v] = smax(ext_s[0][v][lane], ext_s[1][v][lane]);
      umin[v] = smin(ext_s[0][5 + v][lane], ext_s[1][5 + v][lane]);
    }
#pragma unroll 2
    for (int j = fa; j < fb; ++j) {
      const int e = m.cf_list[j];
      const int f = e >= 0 ? e : ~e;
      const double cf0 = sub_rn(m.f_x[f], xc0), cf1 = sub_rn(m.f_x[m.nf + f], xc1), cf2 = sub_rn(m.f_x[2 * m.nf + f], xc2);
#pragma unroll
      for (int v = 0; v < 5; ++v) {
        const double dM = add_rn(add_rn(mul_rn(g[3 * v], cf0), mul_rn(g[3 * v + 1], cf1)), mul_rn(g[3 * v + 2], cf2));
        double dP = u0[v];
        if (dM > 0.) dP = sub_rn(umax[v], dP);
        else if (dM < 0.) dP = sub_rn(umin[v], dP);
        const double dP2 = mul_rn(dP, dP), dM2 = mul_rn(dM, dM);
        if (dM != 0.) {
          const double num = add_rn(add_rn(dP2, eps2[v]), mul_rn(mul_rn(2., dM), dP));
          const double den = add_rn(add_rn(add_rn(dP2, mul_rn(2., dM2)), mul_rn(dM, dP)), eps2[v]);
          phi[v] = smin(phi[v], div_rn(num, den));
        }
      }
    }
#pragma unroll
    for (int v = 0; v < 5; ++v) phi_s[h][v][lane] = phi[v];
    __syncthreads();
#pragma unroll
    for (int v = 0; v < 5; ++v) phi[v] = smin(phi_s[0][v][lane], phi_s[1][v][lane]);
  }
  if (act) {
#pragma unroll
    for (int v = 0; v < 5; ++v)
      if ((h == 0) == (v < 3)) Lm[v * nc + c] = phi[v];
  }
}

// Density the reference's `right` state cache holds when face f is reached:
// the right density of face f-1 (walking back over faces whose BC branch
// does not set it).  Face 0 starts from the zero-initialised cache.
template <class S>
__device__ S cached_right_rho(const DevCase &cs, const DevMesh &m, const S *W, const S *G, const S *Lm, int f) {
  for (int g = f - 1; g >= 0; --g) {
    const double n[3] = {m.f_n[g], m.f_n[m.nf + g], m.f_n[2 * m.nf + g]};
    const double xf[3] = {m.f_x[g], m.f_x[m.nf + g], m.f_x[2 * m.nf + g]};
    const int b = m.f_bc[g];
    if (b < 0) {
      FState<S> R;
      recon_state(cs, m, W, G, Lm, m.f_neighbor[g], xf, R, n);
      return R.rho;
    }
    FState<S> L, R;
    recon_state(cs, m, W, G, Lm, m.f_parent[g], xf, L, n);
    const int gh = m.f_neighbor[g], nt = m.nt;
    R.pc = W[gh]; R.Vc[0] = W[nt + gh]; R.Vc[1] = W[2 * nt + gh]; R.Vc[2] = W[3 * nt + gh]; R.Tc = W[4 * nt + gh];
    R.rho = S(0.);
    if (apply_bc(cs, cs.bc[b], L, R, n, (int *)nullptr)) return R.rho;
  }
  return S(0.);
}

template <class S>
__global__ void k_outlet_rho(DevCase cs, DevMesh m, const S *__restrict__ W, const S *__restrict__ G,
                             const S *__restrict__ Lm, S *__restrict__ stale) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m.n_outlet) return;
  const int f = m.outlet_faces[i];
  stale[m.f_neighbor[f] - m.nc] = cached_right_rho(cs, m, W, G, Lm, f);
}

// ---- convective fluxes in xyz (rotated-frame algebra of ns_roe.cc,
// ns_ausm_plus_up.cc, ns_vanleer.cc, rotated back as in
// ns_convective_face_flux.cc:51-55, per unit area)
template <class S>
__host__ __device__ __forceinline__ void roe(const DevCase &c, const FState<S> &L, const FState<S> &R, const double n[3], S F[5], S &wL) {
  const double G = c.gamma;
  S r = sqrt(R.rho / L.rho);
  const S ir = 1. / (1. + r);
  S Vr[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) Vr[i] = (L.V[i] + r * R.V[i]) * ir;
  const S u = (L.Vn + r * R.Vn) * ir;
  const S H = (L.H + r * R.H) * ir;
  const S a = sqrt((G - 1.) * (H - 0.5 * (Vr[0] * Vr[0] + Vr[1] * Vr[1] + Vr[2] * Vr[2])));
  r = r * L.rho;
  const S Du = R.Vn - L.Vn, Dp = R.p - L.p;
  S lambda, dV, Dl, mdot;
  if (u >= 0.) {
    dV = 0.5 * (Dp - r * a * Du) / (a * a);
    lambda = u - a;
    Dl = 2. * smin(a, smax(S(0.), 2. * (L.a - R.a + Du)));
    if (lambda <= -0.5 * Dl) {
    } else if (lambda < 0.5 * Dl) {
      const S t = lambda - 0.5 * Dl;
      lambda = -0.5 * t * t / Dl;
    } else {
      lambda = S(0.);
    }
    mdot = L.rho * L.Vn;
    const S pr = lambda * dV;
    F[0] = mdot + pr;
#pragma unroll
    for (int i = 0; i < 3; ++i) F[1 + i] = mdot * L.V[i] + L.p * n[i] + pr * (Vr[i] - a * n[i]);
    F[4] = mdot * L.H + pr * (H - u * a);
  } else {
    dV = 0.5 * (Dp + r * a * Du) / (a * a);
    lambda = u + a;
    Dl = 2. * smin(a, smax(S(0.), 2. * (R.a - L.a + Du)));
    if (lambda >= 0.5 * Dl) {
    } else if (lambda > -0.5 * Dl) {
      const S t = lambda + 0.5 * Dl;
      lambda = 0.5 * t * t / Dl;
    } else {
      lambda = S(0.);
    }
    mdot = R.rho * R.Vn;
    const S pr = lambda * dV;
    F[0] = mdot - pr;
#pragma unroll
    for (int i = 0; i < 3; ++i) F[1 + i] = mdot * R.V[i] + R.p * n[i] - pr * (Vr[i] + a * n[i]);
    F[4] = mdot * R.H - pr * (H + u * a);
  }
  wL = S(0.5);
}

template <class S> __host__ __device__ __forceinline__ S m2p(S M) { return 0.25 * (M + 1.) * (M + 1.); }
template <class S> __host__ __device__ __forceinline__ S m2m(S M) { return -0.25 * (M - 1.) * (M - 1.); }

template <class S>
__host__ __device__ __forceinline__ void ausm(const DevCase &c, const FState<S> &L, const FState<S> &R, const double n[3], S F[5], S &wL) {
  const double beta = 0.125, Kp = 0.25, Ku = 0.75, sigma = 1.;
  const S aLh = L.a * L.a / smax(L.a, L.Vn);
  const S aRh = R.a * R.a / smax(R.a, -1. * R.Vn);
  const S a = smin(aLh, aRh);
  const S rho = 0.5 * (L.rho + R.rho);
  const S ML = L.Vn / a, MR = R.Vn / a;
  const S Mbar2 = 0.5 * (ML * ML + MR * MR);
  S Mref = smax(S(c.Minf), sqrt(Mbar2));
  Mref = smin(Mref, S(1.));
  S fa;
  if (Mbar2 >= 1.) fa = S(1.);
  else {
    const S Mo = sqrt(smin(S(1.), smax(Mbar2, Mref * Mref)));
    fa = Mo * (2. - Mo);
  }
  const S m4p = (fabs(ML) >= 1.) ? 0.5 * (ML + fabs(ML)) : m2p(ML) * (1. - 16. * beta * m2m(ML));
  const S m4m = (fabs(MR) >= 1.) ? 0.5 * (MR - fabs(MR)) : m2m(MR) * (1. + 16. * beta * m2p(MR));
  const S M = m4p + m4m - Kp / fa * smax(1. - sigma * Mbar2, S(0.)) * (R.p - L.p) / (rho * a * a);
  const S mdot = (M > 0.) ? a * M * L.rho : a * M * R.rho;
  const S alpha = 3. / 16. * (-4. + 5. * fa * fa);
  const S p5p = (fabs(ML) >= 1.) ? 0.5 * (ML + fabs(ML)) / ML : m2p(ML) * ((2. - ML) - 16. * alpha * ML * m2m(ML));
  const S p5m = (fabs(MR) >= 1.) ? 0.5 * (MR - fabs(MR)) / MR : m2m(MR) * ((-2. - MR) + 16. * alpha * MR * m2p(MR));
  S p = p5p * (L.p + c.Pref) + p5m * (R.p + c.Pref) - Ku * p5p * p5m * (L.rho + R.rho) * fa * a * (R.Vn - L.Vn);
  p = p - c.Pref;
  F[0] = mdot;
  const FState<S> &U = (mdot > 0.) ? L : R;
#pragma unroll
  for (int i = 0; i < 3; ++i) F[1 + i] = mdot * U.V[i] + p * n[i];
  F[4] = mdot * U.H;
  wL = (mdot > 0.) ? S(1.) : S(0.);
}

template <class S>
__host__ __device__ __forceinline__ void vanleer(const DevCase &c, const FState<S> &L, const FState<S> &R, const double n[3], S F[5], S &wL) {
  const double G = c.gamma;
  const S ML = L.Vn / L.a, MR = R.Vn / R.a;
  const S M = 0.5 * (ML + MR);
  if (M <= -1.) {
    const S mdot = R.rho * R.Vn;
    F[0] = mdot;
#pragma unroll
    for (int i = 0; i < 3; ++i) F[1 + i] = mdot * R.V[i] + R.p * n[i];
    F[4] = mdot * R.H;
    wL = S(0.);
  } else if (M >= 1.) {
    const S mdot = L.rho * L.Vn;
    F[0] = mdot;
#pragma unroll
    for (int i = 0; i < 3; ++i) F[1 + i] = mdot * L.V[i] + L.p * n[i];
    F[4] = mdot * L.H;
    wL = S(1.);
  } else {
    const S fp = 0.25 * L.rho * L.a * (ML + 1.) * (ML + 1.);
    const S fm = -0.25 * R.rho * R.a * (1. - MR) * (1. - MR);
    F[0] = fp + fm;
    S tL = (2. * L.a / G) * (0.5 * (G - 1.) * ML + 1.);
    S tR = (2. * R.a / G) * (0.5 * (G - 1.) * MR - 1.);
    const S fn1 = fp * tL + fm * tR - c.Pref;
    S VtL[3], VtR[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) { VtL[i] = L.V[i] - L.Vn * n[i]; VtR[i] = R.V[i] - R.Vn * n[i]; }
#pragma unroll
    for (int i = 0; i < 3; ++i) F[1 + i] = fn1 * n[i] + fp * VtL[i] + fm * VtR[i];
    const double k = 0.5 * G * G / (G * G - 1.);
    tL = k * tL * tL + 0.5 * (VtL[0] * VtL[0] + VtL[1] * VtL[1] + VtL[2] * VtL[2]);
    tR = k * tR * tR + 0.5 * (VtR[0] * VtR[0] + VtR[1] * VtR[1] + VtR[2] * VtR[2]);
    F[4] = fp * tL + fm * tR;
    wL = S(0.5);
  }
}

// SD-SLAU (ns_sd_slau.cc:37-94) in xyz.  alpha = 0 (ns_sd_slau.cc:47)
// removes the alpha terms of B+ and B-.  The pressure sensor theta
// (ns_sd_slau.cc:68-71) is identically 1: max_delta_p is |delta_p| itself
// (ns_sd_slau.cc:64), so with x = |delta_p| / p_ave >= 0 the ratio
// (Csd2 x + Csd1) / (x + Csd1), Csd2 = 10 > 1, is >= 1 after rounding too
// (every step is monotone) and min(1, theta^2) returns the constant 1 for every
// state with positive absolute pressure.  The speed-of-sound scale keeps the
// reference's Mhat = min(1, sqrt(0.5 (|V_L|^2 + |V_R|^2) / a)) (a, not a^2).
template <class S>
__host__ __device__ __forceinline__ void sdslau(const DevCase &c, const FState<S> &L, const FState<S> &R, const double n[3], S F[5], S &wL) {
  const S a = 0.5 * (L.a + R.a);
  const S qL = L.V[0] * L.V[0] + L.V[1] * L.V[1] + L.V[2] * L.V[2];
  const S qR = R.V[0] * R.V[0] + R.V[1] * R.V[1] + R.V[2] * R.V[2];
  const S Mhat = smin(S(1.), S(sqrt(0.5 * (qL + qR) / a)));
  const S chi = (1. - Mhat) * (1. - Mhat);
  const S Mp = L.Vn / a, Mm = R.Vn / a;
  const S Bp = (fabs(Mp) < 1.) ? S(0.25 * (2. - Mp) * (Mp + 1.) * (Mp + 1.)) : S((Mp > 0.) ? 1. : 0.);
  const S Bm = (fabs(Mm) < 1.) ? S(0.25 * (2. + Mm) * (Mm - 1.) * (Mm - 1.)) : S((Mm < 0.) ? 1. : 0.);
  const S pave = 0.5 * (L.p + R.p) + c.Pref;
  const S dp = R.p - L.p;
  S p = pave - 0.5 * (Bp - Bm) * dp + (1. - chi) * (Bp + Bm - 1.) * pave;
  const S g = -smax(smin(Mp, S(0.)), S(-1.)) * smin(smax(Mm, S(0.)), S(1.));
  const S aL = fabs(L.Vn), aR = fabs(R.Vn);
  const S Vn = (L.rho * aL + R.rho * aR) / (L.rho + R.rho);
  const S Vp = (1. - g) * Vn + g * aL;
  const S Vm = (1. - g) * Vn + g * aR;
  const S mdot = 0.5 * (L.rho * (L.Vn + Vp) + R.rho * (R.Vn - Vm) - smax(S(0.), S(1. - Vn / a)) * dp / a);
  p = p - c.Pref;
  F[0] = mdot;
  const FState<S> &U = (mdot > 0.) ? L : R;
#pragma unroll
  for (int i = 0; i < 3; ++i) F[1 + i] = mdot * U.V[i] + p * n[i];
  F[4] = mdot * U.H;
  wL = (mdot > 0.) ? S(1.) : S(0.);
}

// sqrt(x^2 + e^2) whose tangent is 0 where the value is 0 (|x| at x = e = 0
// has no derivative; the value is the reference's)
template <class S>
__host__ __device__ __forceinline__ S hypot0(const S &q) {
  return (q == 0.) ? S(0.) : S(sqrt(q));
}

// Steger-Warming flux-vector splitting with wall dissipation
// (Stegger_Warming_flux, ns_stegger_warming.cc:23-145) in xyz.  Per signal
// the reference forms Jacob = L diag(Lambda) R in the rotated frame at the
// w-weighted state and adds Jacob Q of the upwind side.  Here the product is
// applied right to left and the rotated rows are written with frame-free
// vectors (u = weighted velocity, m = rho V of the upwind side, un = u.n):
//   r0 = (a^2 - gs) Q0 + beta (u.m - Q4),  r3,4 = (gs -+ un a) Q0 +- a (m.n) - beta (u.m - Q4),
//   rows 1-2 = the tangential part of d = m - u Q0,
// then with s_k = Lambda_k r_k and st = Lambda_0 (d - n (d.n)):
//   F0 = c,  Fm = c u + 0.5 a (s3 - s4) / a^2 n + st,
//   F4 = eta s0 + u.st + 0.5 (H (s3 + s4) + a un (s3 - s4)) / a^2,
//   c = (s0 + 0.5 (s3 + s4)) / a^2.
// The pressure and temperature enter as stored (gauge values, as in the
// reference); weightL ends as w, the value the second pass leaves.
template <class S>
__host__ __device__ __forceinline__ void sw(const DevCase &c, const FState<S> &L, const FState<S> &R, const double n[3],
                                            double diss, double wall_d, S F[5], S &wL) {
  const double alpha = 6.;
  const double beta = c.gamma * c.R / c.Cp;
  const S dpr = fabs(L.p - R.p) / smin(L.p, R.p);
  const S w = 0.5 / (alpha * alpha * dpr * dpr + 1.);
#pragma unroll
  for (int k = 0; k < 5; ++k) F[k] = S(0.);
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const double sg = h ? -1. : 1.;
    const S wl = h ? w : S(1. - w);
    const S wr = 1. - wl;
    const S p = wl * L.p + wr * R.p;
    S u[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) u[i] = wl * L.V[i] + wr * R.V[i];
    const S V2 = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
    const S un = u[0] * n[0] + u[1] * n[1] + u[2] * n[2];
    const S T = wl * L.T + wr * R.T;
    const S rho = wl * L.rho + wr * R.rho;
    const S a2 = (1. + beta) * p / rho;
    const S a = sqrt(a2);
    const S H = 0.5 * V2 + a2 / (c.gamma - 1.);
    const S gs = c.R * T + beta * (0.5 * V2 - c.Cp * T / c.gamma);
    const S eta = (beta * V2 - gs) / (beta * a2);
    const S eps = (wall_d > c.bl_height) ? S(c.wdiss * (a + hypot0(V2))) : S(c.wdiss * diss * (a + fabs(un)));
    const S e2 = eps * eps;
    const S l0 = 0.5 * (un + sg * hypot0(S(un * un + e2)));
    const S up = un + a, um = un - a;
    const S l3 = 0.5 * (up + sg * hypot0(S(up * up + e2)));
    const S l4 = 0.5 * (um + sg * hypot0(S(um * um + e2)));
    const FState<S> &U = h ? R : L;
    const S Q0 = U.rho, Q4 = U.rho * U.H - U.p;
    S mm[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) mm[i] = U.rho * U.V[i];
    const S um_ = u[0] * mm[0] + u[1] * mm[1] + u[2] * mm[2];
    const S mn = mm[0] * n[0] + mm[1] * n[1] + mm[2] * n[2];
    const S bq = beta * (um_ - Q4);
    const S s0 = l0 * ((a2 - gs) * Q0 + bq);
    const S s3 = l3 * ((gs - un * a) * Q0 + a * mn - bq);
    const S s4 = l4 * ((gs + un * a) * Q0 - a * mn - bq);
    S d[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) d[i] = mm[i] - u[i] * Q0;
    const S dn = d[0] * n[0] + d[1] * n[1] + d[2] * n[2];
    S st[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) st[i] = l0 * (d[i] - dn * n[i]);
    const S cc = (s0 + 0.5 * (s3 + s4)) / a2;
    const S cn = 0.5 * a * (s3 - s4) / a2;
    F[0] = F[0] + cc;
#pragma unroll
    for (int i = 0; i < 3; ++i) F[1 + i] = F[1 + i] + cc * u[i] + cn * n[i] + st[i];
    F[4] = F[4] + eta * s0 + (u[0] * st[0] + u[1] * st[1] + u[2] * st[2]) + 0.5 * (H * (s3 + s4)) / a2 + un * cn;
  }
  wL = w;
}

// Sources of the u, v, w, T gradient rows (12 values per cell) that the
// viscous flux reads: the stored cell gradients, or local copies (adjoint
// kernels, where they are independent inputs).
template <class SG>
struct GlobalGrad {
  typedef SG value_type;
  const SG *G;
  int nc, pa, nb;
  __device__ __forceinline__ SG at_pa(int i) const { return G[(3 + i) * nc + pa]; }
  __device__ __forceinline__ SG at_nb(int i) const { return G[(3 + i) * nc + nb]; }
};
template <class SG>
struct LocalGrad {
  typedef SG value_type;
  const SG *gpa, *gnb;
  __device__ __forceinline__ SG at_pa(int i) const { return gpa[i]; }
  __device__ __forceinline__ SG at_nb(int i) const { return gnb[i]; }
};

// Face difference D = F_diffusive - F_convective * A for prepared left/right
// states (convective_face_flux + diffusive_face_flux,
// ns_convective_face_flux.cc:32-59, ns_diffusive_face_flux.cc:28-64).  GS
// supplies the parent / neighbour gradient rows (GlobalGrad or LocalGrad);
// its value type is S itself, or double when only the face states carry
// tangents, as in the face-Jacobian kernel.
//
// FX selects the convective flux at compile time: 0 = Roe / Van Leer /
// AUSM+up chosen at run time by cs.flux (ns.h:48-53 numbering), 4 = SD-SLAU,
// 5 = Steger-Warming.  Kernels are instantiated per selector (FCFD_BY_FLUX)
// so the larger SD-SLAU and Steger-Warming bodies add no registers to the
// other fluxes' kernels.
//
// mu_t: the face eddy viscosities, indexed by face (null: laminar); MT is a
// pointer, or a view whose operator[] gives the face's value (the adjoint's
// seeded input).
template <class S, class GS, bool VISCOUS, int FX, class MT = const typename GS::value_type *>
__device__ __forceinline__ void face_D(const DevCase &cs, const DevMesh &m, int f, const double n[3], double A, int b,
                                       int pa, int nb, const FState<S> &L, const FState<S> &R, const GS &gs,
                                       MT mu_t, S D[5], S &wL) {
  const int nf = m.nf, nt = m.nt;
  S F[5];
  if (FX == 4) sdslau(cs, L, R, n, F, wL);
  else if (FX == 5) sw(cs, L, R, n, m.f_diss[f], m.f_wall[f], F, wL);
  else if (cs.flux == 1) roe(cs, L, R, n, F, wL);
  else if (cs.flux == 2) vanleer(cs, L, R, n, F, wL);
  else ausm(cs, L, R, n, F, wL);
  S Fd[5] = {S(0.), S(0.), S(0.), S(0.), S(0.)};
  if (VISCOUS) {
    // face_state_update (ns_assemble_linear_system.cc:353-415)
    S gr[12];  // u,v,w,T gradients at the face
    if (b >= 0) {
#pragma unroll
      for (int i = 0; i < 12; ++i) gr[i] = S(gs.at_pa(i));
    } else {
      const double wP = m.f_w[f], wN = m.f_w[nf + f];
#pragma unroll
      for (int i = 0; i < 12; ++i) gr[i] = S(wP * gs.at_pa(i) + wN * gs.at_nb(i));
    }
    const double l0 = m.c_x[nb] - m.c_x[pa], l1 = m.c_x[nt + nb] - m.c_x[nt + pa], l2 = m.c_x[2 * nt + nb] - m.c_x[2 * nt + pa];
    const double ilm = 1. / sqrt(l0 * l0 + l1 * l1 + l2 * l2);
    const double e0 = l0 * ilm, e1 = l1 * ilm, e2 = l2 * ilm;
    const S dc[4] = {R.Vc[0] - L.Vc[0], R.Vc[1] - L.Vc[1], R.Vc[2] - L.Vc[2], R.Tc - L.Tc};
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const S dn = gr[3 * q] * e0 + gr[3 * q + 1] * e1 + gr[3 * q + 2] * e2;
      const S s = dc[q] * ilm - dn;
      gr[3 * q] = gr[3 * q] + s * e0;
      gr[3 * q + 1] = gr[3 * q + 1] + s * e1;
      gr[3 * q + 2] = gr[3 * q + 2] + s * e2;
    }
    const S Vf[3] = {0.5 * (L.V[0] + R.V[0]), 0.5 * (L.V[1] + R.V[1]), 0.5 * (L.V[2] + R.V[2])};
    const S Tf = 0.5 * (L.T + R.T);
    S mu = viscosity(cs, Tf);
    S lam = cs.prandtl ? cs.Cp * mu / cs.Pr : S(cs.lambda);  // therm_cond without a second viscosity
    if (mu_t) {
      const S mt = S(mu_t[f]);
      mu = mu + mt;
      lam = lam + cs.Cp * mt / cs.Pr_t;
    }
    const S *gu = gr, *gv = gr + 3, *gw = gr + 6, *gT = gr + 9;
    const S tx0 = 2. / 3. * (2. * gu[0] - gv[1] - gw[2]), tx1 = gu[1] + gv[0], tx2 = gu[2] + gw[0];
    const S ty1 = 2. / 3. * (2. * gv[1] - gu[0] - gw[2]), ty2 = gv[2] + gw[1];
    const S tz2 = 2. / 3. * (2. * gw[2] - gu[0] - gv[1]);
    const double an[3] = {n[0] * A, n[1] * A, n[2] * A};
    Fd[1] = mu * (tx0 * an[0] + tx1 * an[1] + tx2 * an[2]);
    Fd[2] = mu * (tx1 * an[0] + ty1 * an[1] + ty2 * an[2]);
    Fd[3] = mu * (tx2 * an[0] + ty2 * an[1] + tz2 * an[2]);
    Fd[4] = mu * ((tx0 * Vf[0] + tx1 * Vf[1] + tx2 * Vf[2]) * an[0] + (tx1 * Vf[0] + ty1 * Vf[1] + ty2 * Vf[2]) * an[1] +
                  (tx2 * Vf[0] + ty2 * Vf[1] + tz2 * Vf[2]) * an[2]);
    S qq = lam * (gT[0] * an[0] + gT[1] * an[1] + gT[2] * an[2]);
    if (b >= 0 && cs.bc[b].thermal == TH_FIXED_Q_) qq = S(cs.bc[b].qdot * A);
    Fd[4] = Fd[4] + qq;
  }
#pragma unroll
  for (int v = 0; v < 5; ++v) D[v] = Fd[v] - F[v] * A;
}

// Left / right states of face f (reconstruction, or the boundary condition
// with the cached density where the BC branch leaves it untouched).  STALE:
// 0 reads the cached density from `stale`; 1 returns false instead (the face
// is left to the outlet kernel); 2 computes it here (the walk back of
// cached_right_rho) and stores it in `stale`.  Returns true when the states
// are complete.
template <class S, int STALE = 0, class SA = S>
__device__ __forceinline__ bool face_states(const DevCase &cs, const DevMesh &m, int f, const double n[3], int b, int pa,
                                            int nb, const SA *__restrict__ W, const SA *__restrict__ G, const SA *__restrict__ Lm,
                                            S *stale, FState<S> &L, FState<S> &R, int *err) {
  const int nf = m.nf, nt = m.nt, nc = m.nc;
  const double xf[3] = {m.f_x[f], m.f_x[nf + f], m.f_x[2 * nf + f]};
  recon_state<S, SA>(cs, m, W, G, Lm, pa, xf, L, n);
  if (b < 0) {
    recon_state<S, SA>(cs, m, W, G, Lm, nb, xf, R, n);
  } else {
    R.pc = W[nb]; R.Vc[0] = W[nt + nb]; R.Vc[1] = W[2 * nt + nb]; R.Vc[2] = W[3 * nt + nb]; R.Tc = W[4 * nt + nb];
    R.rho = S(0.);
    if (!apply_bc(cs, cs.bc[b], L, R, n, err)) {
      if (STALE == 1) return false;
      if (STALE == 2) {
        R.rho = cached_right_rho(cs, m, W, G, Lm, f);
        stale[nb - nc] = R.rho;
      } else {
        R.rho = stale[nb - nc];
      }
    } else if (STALE == 2) {
      return false;
    }
    finish(cs, R, n);
  }
  return true;
}

// Face flux: reconstruction, BCs, inviscid + viscous flux; D = Fd - Fc.
// OUTLET = false: every face except the outlet faces whose BC branch leaves
// the right density to the state cache; OUTLET = true: those faces only
// (thread i takes outlet face i), with the cached density computed in place
// and stored in `stale` for the face-Jacobian kernel.  The two launches write
// disjoint faces and run concurrently.
template <class S, bool VISCOUS, int FX, bool OUTLET, bool PART = false>
__global__ void __launch_bounds__(128) k_face_flux(DevCase cs, DevMesh m, const S *__restrict__ W, const S *__restrict__ G,
                                                   const S *__restrict__ Lm, S *stale,
                                                   const S *__restrict__ mu_t, S *__restrict__ D, S *__restrict__ mdot_out,
                                                   S *__restrict__ wl_out, int *err) {
  pdl_wait();
  pdl_trigger();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int nf = m.nf;
  // main launch: face_list when viscous (faces grouped by kind: an interior
  // viscous face costs several boundary faces, so mixed warps would run both
  // paths) or partitioned, else face order (inviscid faces are cheap enough
  // that the coalesced face arrays matter more); outlet launch: all outlet
  // faces, or (PART) one rank's
  int f;
  if constexpr (OUTLET) {
    if constexpr (PART) {
      if (i >= m.n_part_outlet) return;
      f = m.outlet_faces[m.part_outlet[i]];
    } else {
      if (i >= m.n_outlet) return;
      f = m.outlet_faces[i];
    }
  } else if constexpr (VISCOUS || PART) {
    if (i >= m.n_face_list) return;
    f = m.face_list[i];
  } else {
    if (i >= nf) return;
    f = i;
  }
  const int pa = m.f_parent[f], nb = m.f_neighbor[f], b = m.f_bc[f];
  const double n[3] = {m.f_n[f], m.f_n[nf + f], m.f_n[2 * nf + f]};
  const double A = m.f_area[f];
  FState<S> L, R;
  if (!face_states<S, OUTLET ? 2 : 1>(cs, m, f, n, b, pa, nb, W, G, Lm, stale, L, R, err)) return;
  S Dv[5], wL;
  const GlobalGrad<S> gs{G, m.nc, pa, nb};
  face_D<S, GlobalGrad<S>, VISCOUS, FX>(cs, m, f, n, A, b, pa, nb, L, R, gs, mu_t, Dv, wL);
#pragma unroll
  for (int v = 0; v < 5; ++v) D[v * nf + f] = Dv[v];
  if (mdot_out) mdot_out[f] = (-Dv[0]) / A;
  if (wl_out) wl_out[f] = wL;
}

// Initial values of the extrema slots (even: max, starts at key 0; odd: min,
// starts at all ones) and of the first-attaining-cell slots.
__device__ __forceinline__ void reset_extrema(unsigned long long *ext, int *argx) {
  const int t = threadIdx.x;
  if (blockIdx.x == 0 && t < 8) {
    if (ext) ext[t] = (t & 1) ? ~0ull : 0ull;
    if (argx) argx[t] = 0x7F7F7F7F;
  }
}

// Atomic-free gather: R_c = sum over the cell's faces in ascending face order
// of (+D) for the parent side and (-D) for the neighbour side.  The last
// kernel of a residual chain, so it also re-arms the extrema slots for the
// next chain (every reader of them has finished by now on this stream).
template <class S, bool AOS>
__global__ void k_gather(DevMesh m, const S *__restrict__ D, S *__restrict__ R, unsigned long long *ext, int *argx) {
  pdl_wait();
  reset_extrema(ext, argx);
  // one thread per (cell, equation): 5 nc threads, equation-major so that a
  // warp covers consecutive cells of one equation
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int nc = m.nc, no = n_owned(m), lo = m.part_cells ? m.own_lo : 0;
  if (t >= 5 * no) return;
  const int v = t / no, c = lo + (t - v * no);
  const S *Dv = D + (size_t)v * m.nf;
  const int j0 = m.cf_index[c], j1 = m.cf_index[c + 1];
  S r = S(0.);
  int j = j0;
  // face ids first (up to 6 at once), then the D values, summed in ascending
  // face order
  for (; j + 6 <= j1; j += 6) {
    int e[6];
#pragma unroll
    for (int q = 0; q < 6; ++q) e[q] = m.cf_list[j + q];
    S d[6];
#pragma unroll
    for (int q = 0; q < 6; ++q) d[q] = Dv[e[q] >= 0 ? e[q] : ~e[q]];
#pragma unroll
    for (int q = 0; q < 6; ++q) r = r + ((e[q] >= 0 ? d[q] : -1. * d[q]) + 0.);
  }
  for (; j < j1; ++j) {
    const int e = m.cf_list[j];
    if (e >= 0) r = r + (Dv[e] + 0.);
    else r = r + (-1. * Dv[~e] + 0.);
  }
  if (AOS) R[5 * c + v] = r;
  else R[(size_t)v * nc + c] = r;
}

// Local time step (time_step.cc:143-224).
template <class S>
__global__ void k_local_dt(DevCase cs, DevMesh m, const S *__restrict__ W, S *__restrict__ dt, double cfl,
                           unsigned long long *__restrict__ minkey) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= m.nc) return;
  const int nt = m.nt;
  const S p = W[c], u = W[nt + c], v = W[2 * nt + c], w = W[3 * nt + c], T = W[4 * nt + c];
  const S a = sound(cs, p, T);
  const S v_dt = cfl * m.c_len[c] / (sqrt(u * u + v * v + w * w) + a);
  dt[c] = v_dt;
  // a NaN step drops out of the minimum, as it does in update_time_step's
  // std::min (time_step.cc:181-186)
  if (minkey && val(v_dt) == val(v_dt)) atomicMin(minkey, okey(val(v_dt)));
}

template <class S>
__global__ void k_fill_min(int n, S *__restrict__ dt, const unsigned long long *__restrict__ minkey) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < n) dt[c] = S(okey_inv(*minkey));
}

}  // namespace fcfd
