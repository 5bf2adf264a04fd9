// Adjoint (vector-Jacobian product) of the residual, and the boundary-load
// functional with its state gradient.
//
//   fcfd_vjp:   Wbar = (dR/dW)^T Rbar
//   fcfd_drag:  F = sum over the selected BC regions' faces of the
//               convective-minus-diffusive momentum flux (the loads of
//               ns_assemble_linear_system.cc:108-119), J = F . dir and dJ/dW.
//
// The forward chain (ghost update, LSQ gradient, limiter, face flux, gather)
// is reversed stage by stage, with the nonlinear local maps differentiated by
// multi-lane forward duals and then transposed:
//   1. face stage: per face, the face difference D_f as a function of its 45
//      local inputs (reconstructed left/right states, cell-centre states, the
//      stale right density, the viscous gradient rows) is differentiated lane
//      by lane and contracted with Dbar_f (from Rbar by the gather's transpose,
//      or from the load seed): the input adjoints are recomputed per face, not
//      stored as Jacobians;
//   2. stale-density stage: outlet faces that read the previous face's right
//      density pass their adjoint back to that face;
//   3. cell stage: per cell, the face-input adjoints are gathered in ascending
//      face order and pushed through the reconstruction W + Lm (G . d), giving
//      the cell's state, gradient and limiter adjoints; the limiter adjoint
//      follows the face that attained the minimum (VK, minmod, BJ) into the
//      cell state, its gradient, the neighbour that held the extreme value and
//      the global VK extrema;
//   4. gradient stage: the LSQ map G_c = sum_k w_ck W_k transposed as a gather
//      over the transposed stencil (deterministic);
//   5. ghost stage: ghost states are the first-order boundary update of the
//      parent cell, differentiated per boundary face and gathered per cell.
// Every accumulation has a fixed order, so Wbar is the same bits on every run:
// limiter-neighbour contributions are written per (variable, face, side) and
// gathered per cell in face order, the outlet faces' stale-density adjoints are
// summed per target face in outlet order, and the global extrema's adjoints go
// through per-block partial sums added by one block.
#include <algorithm>
#include <cmath>
#include <vector>

#include "ctx.hpp"
#include "dn.cuh"
#include "kw.cuh"

namespace fcfd {

extern template __global__ void k_ghost_minmax<double>(DevCase, DevMesh, double *, unsigned long long *, int *);

namespace {

constexpr int kLanes = 4;
typedef DN<kLanes> DA;

// local face inputs (U_MUT: the face eddy viscosity of a turbulent case)
enum { U_QL = 0, U_CL = 5, U_QR = 10, U_CR = 15, U_STALE = 20, U_GPA = 21, U_GNB = 33, U_MUT = 45, U_N = 46 };

// seeded view of a face's local inputs for one pass: input i carries lane l
// when chunk[l] == i
struct Seeds {
  const double *u;
  int chunk[kLanes];
  __device__ __forceinline__ DA operator()(int i) const {
    DA r(u[i]);
#pragma unroll
    for (int l = 0; l < kLanes; ++l)
      if (chunk[l] == i) r.d[l] = 1.;
    return r;
  }
};
struct SeedGrad {
  typedef DA value_type;
  const Seeds *s;
  __device__ __forceinline__ DA at_pa(int i) const { return (*s)(U_GPA + i); }
  __device__ __forceinline__ DA at_nb(int i) const { return (*s)(U_GNB + i); }
};
// the face eddy viscosity as face_D reads it (mu_t[f]); off for laminar cases
struct SeedMut {
  DA v;
  bool on;
  __device__ __forceinline__ DA operator[](int) const { return v; }
  __device__ __forceinline__ explicit operator bool() const { return on; }
};

template <class F>
__device__ __forceinline__ void state_from(const DevCase &cs, FState<DA> &s, const F &in, int q, int cc, const double n[3]) {
  s.p = in(q); s.V[0] = in(q + 1); s.V[1] = in(q + 2); s.V[2] = in(q + 3); s.T = in(q + 4);
  s.pc = in(cc); s.Vc[0] = in(cc + 1); s.Vc[1] = in(cc + 2); s.Vc[2] = in(cc + 3); s.Tc = in(cc + 4);
  s.rho = eos_rho(cs, s.p, s.T);
  finish(cs, s, n);
}

// D_f, the left weight and the right density of face f from its local
// inputs (the same sequence as face_states + face_D); turb: the face eddy
// viscosity is an input.
template <bool VISCOUS, int FX>
__device__ void face_from_inputs(const DevCase &cs, const DevMesh &m, int f, const double n[3], double A, int b, int pa,
                                 int nb, bool turb, const Seeds &in, DA D[5], DA &wL, DA &rhoR) {
  FState<DA> L, R;
  state_from(cs, L, in, U_QL, U_CL, n);
  if (b < 0) {
    state_from(cs, R, in, U_QR, U_CR, n);
  } else {
    R.pc = in(U_CR); R.Vc[0] = in(U_CR + 1); R.Vc[1] = in(U_CR + 2); R.Vc[2] = in(U_CR + 3); R.Tc = in(U_CR + 4);
    R.rho = DA(0.);
    if (!apply_bc(cs, cs.bc[b], L, R, n, (int *)nullptr)) R.rho = in(U_STALE);
    finish(cs, R, n);
  }
  rhoR = R.rho;
  const SeedGrad gs{&in};
  const SeedMut mt{turb ? in(U_MUT) : DA(0.), turb};
  face_D<DA, SeedGrad, VISCOUS, FX, SeedMut>(cs, m, f, n, A, b, pa, nb, L, R, gs, mt, D, wL);
}

// Forward values of face f's local inputs.
__device__ void face_inputs(const DevMesh &m, int f, int b, int pa, int nb, const double *W, const double *G,
                            const double *Lm, const double *stale, const double *mutf, double u[U_N]) {
  const int nt = m.nt, nc = m.nc, nf = m.nf;
  const double xf[3] = {m.f_x[f], m.f_x[nf + f], m.f_x[2 * nf + f]};
  for (int i = 0; i < U_N; ++i) u[i] = 0.;
  auto recon = [&](int k, int q) {
    const double d0 = xf[0] - m.c_x[k], d1 = xf[1] - m.c_x[nt + k], d2 = xf[2] - m.c_x[2 * nt + k];
    for (int v = 0; v < 5; ++v) {
      const double dot = d0 * G[(3 * v) * nc + k] + d1 * G[(3 * v + 1) * nc + k] + d2 * G[(3 * v + 2) * nc + k];
      u[q + v] = W[v * nt + k] + Lm[v * nc + k] * dot;
    }
  };
  recon(pa, U_QL);
  for (int v = 0; v < 5; ++v) u[U_CL + v] = W[v * nt + pa];
  if (b < 0) recon(nb, U_QR);
  for (int v = 0; v < 5; ++v) u[U_CR + v] = W[v * nt + nb];
  if (b >= 0) u[U_STALE] = stale[nb - nc];
  for (int i = 0; i < 12; ++i) u[U_GPA + i] = G[(3 + i) * nc + pa];
  if (b < 0)
    for (int i = 0; i < 12; ++i) u[U_GNB + i] = G[(3 + i) * nc + nb];
  if (mutf) u[U_MUT] = mutf[f];
}

// Inputs that can influence D_f (or the right density) for this face.
template <bool VISCOUS>
__device__ int active_inputs(const DevCase &cs, int b, bool turb, int act[U_N]) {
  int na = 0;
  for (int i = 0; i < 5; ++i) act[na++] = U_QL + i;
  if (b < 0) for (int i = 0; i < 5; ++i) act[na++] = U_QR + i;
  if (VISCOUS || b >= 0) for (int i = 0; i < 5; ++i) act[na++] = U_CL + i;
  if (VISCOUS) for (int i = 0; i < 5; ++i) act[na++] = U_CR + i;
  if (b >= 0 && (cs.bc[b].type == T_OUTLET || cs.bc[b].type == T_INLET)) act[na++] = U_STALE;
  if (VISCOUS) {
    for (int i = 0; i < 12; ++i) act[na++] = U_GPA + i;
    if (b < 0) for (int i = 0; i < 12; ++i) act[na++] = U_GNB + i;
    if (turb) act[na++] = U_MUT;
  }
  return na;
}

// Limiter-extreme adjoints of each interior cell: the contributions its face
// neighbours left across the shared faces (k_cell_adj's Wface, side 0 = from
// the parent, side 1 = from the neighbour), summed in the cell's ascending
// face order.  Writes Wlim of the interior cells; ghost entries stay zero.
__global__ void k_wlim_gather(DevMesh m, const double *__restrict__ Wface, double *__restrict__ Wlim) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int nc = m.nc, nf = m.nf;
  if (t >= 5 * nc) return;
  const int v = t / nc, c = t - v * nc;
  double acc = 0.;
  for (int j = m.cf_index[c]; j < m.cf_index[c + 1]; ++j) {
    const int e = m.cf_list[j];
    // c is the parent of face e: the neighbour's contribution (side 1);
    // c is the neighbour of face ~e: the parent's (side 0)
    acc += e >= 0 ? Wface[((size_t)v * 2 + 1) * nf + e] : Wface[((size_t)v * 2) * nf + ~e];
  }
  Wlim[(size_t)v * m.nt + c] = acc;
}

// Face stage: FA[i][f] = sum_v Dbar_v dD_v/du_i (+ wLbar dwL/du_i).  A
// turbulent case adds the face eddy viscosity mutf as an input and seeds,
// from the k-omega faces, the adjoints of the face's mass flux mdot = -D_0/A
// (mdotb) and left weight (wlb).
template <bool VISCOUS, int FX>
__global__ void __launch_bounds__(128) k_face_adj(DevCase cs, DevMesh m, const double *__restrict__ W,
                                                  const double *__restrict__ G, const double *__restrict__ Lm,
                                                  const double *__restrict__ stale, const double *__restrict__ Rbar,
                                                  unsigned int load_mask, double dir0, double dir1, double dir2,
                                                  const double *__restrict__ mutf, const double *__restrict__ mdotb,
                                                  const double *__restrict__ wlb, double *__restrict__ FA) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  const int nf = m.nf, nc = m.nc;
  if (f >= nf) return;
  const int pa = m.f_parent[f], nb = m.f_neighbor[f], b = m.f_bc[f];
  const double A = m.f_area[f];
  double Db[5] = {0., 0., 0., 0., 0.};
  if (Rbar) {
    for (int v = 0; v < 5; ++v) Db[v] = Rbar[v * nc + pa] - (b < 0 ? Rbar[v * nc + nb] : 0.);
  }
  if (b >= 0 && ((load_mask >> b) & 1u)) { Db[1] -= dir0; Db[2] -= dir1; Db[3] -= dir2; }
  if (mdotb) Db[0] -= mdotb[f] / A;
  const double wb = wlb ? wlb[f] : 0.;
  const bool turb = mutf != nullptr;
  double ub[U_N];
  for (int i = 0; i < U_N; ++i) ub[i] = 0.;
  if (Db[0] != 0. || Db[1] != 0. || Db[2] != 0. || Db[3] != 0. || Db[4] != 0. || wb != 0.) {
    const double n[3] = {m.f_n[f], m.f_n[nf + f], m.f_n[2 * nf + f]};
    double u[U_N];
    face_inputs(m, f, b, pa, nb, W, G, Lm, stale, mutf, u);
    int act[U_N];
    const int na = active_inputs<VISCOUS>(cs, b, turb, act);
    for (int k0 = 0; k0 < na; k0 += kLanes) {
      Seeds in;
      in.u = u;
      for (int l = 0; l < kLanes; ++l) in.chunk[l] = (k0 + l < na) ? act[k0 + l] : -1;
      DA D[5], wL, rhoR;
      face_from_inputs<VISCOUS, FX>(cs, m, f, n, A, b, pa, nb, turb, in, D, wL, rhoR);
      for (int l = 0; l < kLanes; ++l) {
        if (in.chunk[l] < 0) continue;
        double s = 0.;
        for (int v = 0; v < 5; ++v) s += Db[v] * D[v].d[l];
        if (wb != 0.) s += wb * wL.d[l];
        ub[in.chunk[l]] = s;
      }
    }
  }
  for (int i = 0; i < U_N; ++i) FA[(size_t)i * nf + f] = ub[i];
}

// Stale-density stage: an outlet face that read the right density of an
// earlier face (cached_right_rho) hands that adjoint to the earlier face.
template <bool VISCOUS, int FX>
__global__ void k_stale_adj(DevCase cs, DevMesh m, const double *__restrict__ W, const double *__restrict__ G,
                            const double *__restrict__ Lm, const double *__restrict__ stale, const double *__restrict__ mutf,
                            const double *__restrict__ FA, double *__restrict__ SC, int *__restrict__ tgt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m.n_outlet) return;
  const int nf = m.nf;
  const int f = m.outlet_faces[i];
  const double sb = FA[(size_t)U_STALE * nf + f];
  // walk back exactly as cached_right_rho does; the target is recorded even
  // when this face's seed is zero, so that faces sharing a target stay one run
  for (int g = f - 1; g >= 0; --g) {
    const double n[3] = {m.f_n[g], m.f_n[nf + g], m.f_n[2 * nf + g]};
    const double A = m.f_area[g];
    const int pa = m.f_parent[g], nb = m.f_neighbor[g], b = m.f_bc[g];
    bool sets = true;
    if (b >= 0) {
      FState<double> L, R;
      const double xf[3] = {m.f_x[g], m.f_x[nf + g], m.f_x[2 * nf + g]};
      recon_state(cs, m, W, G, Lm, pa, xf, L, n);
      const int nt = m.nt;
      R.pc = W[nb]; R.Vc[0] = W[nt + nb]; R.Vc[1] = W[2 * nt + nb]; R.Vc[2] = W[3 * nt + nb]; R.Tc = W[4 * nt + nb];
      R.rho = 0.;
      sets = apply_bc(cs, cs.bc[b], L, R, n, (int *)nullptr);
    }
    if (!sets) continue;
    tgt[i] = g;
    if (sb == 0.) return;
    double u[U_N];
    face_inputs(m, g, b, pa, nb, W, G, Lm, stale, mutf, u);
    int act[U_N];
    // the right density does not depend on the eddy viscosity
    const int na = active_inputs<VISCOUS>(cs, b, false, act);
    for (int k0 = 0; k0 < na; k0 += kLanes) {
      Seeds in;
      in.u = u;
      for (int l = 0; l < kLanes; ++l) in.chunk[l] = (k0 + l < na) ? act[k0 + l] : -1;
      DA D[5], wL, rhoR;
      face_from_inputs<VISCOUS, FX>(cs, m, g, n, A, b, pa, nb, mutf != nullptr, in, D, wL, rhoR);
      for (int l = 0; l < kLanes; ++l)
        if (in.chunk[l] >= 0) SC[(size_t)in.chunk[l] * m.n_outlet + i] = sb * rhoR.d[l];
    }
    return;
  }
}

// Adds the outlet faces' stale-density adjoints to the faces whose right
// density they read.  Outlet faces are in ascending face order and so are
// their targets (the last earlier face that sets the density), so the faces
// sharing a target form one contiguous run: its first thread sums the run in
// order and is the only writer of that target's adjoints (deterministic).
__global__ void k_stale_apply(int n_outlet, int nf, const double *__restrict__ SC, const int *__restrict__ tgt,
                              double *__restrict__ FA) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_outlet) return;
  const int g = tgt[i];
  if (g < 0 || (i > 0 && tgt[i - 1] == g)) return;
  int j1 = i + 1;
  while (j1 < n_outlet && tgt[j1] == g) ++j1;
  for (int k = 0; k < U_N; ++k) {
    double acc = 0.;
    for (int j = i; j < j1; ++j) acc += SC[(size_t)k * n_outlet + j];
    if (acc != 0.) FA[(size_t)k * nf + g] += acc;
  }
}

// One face's limiter ratio for variable v as a function of the lanes
// (u0, g0, g1, g2, x, e2); x is the neighbour extreme (VK, BJ) or the
// neighbour value (minmod).  Mirrors k_grad_limiter's per-face expression.
template <class S>
__device__ __forceinline__ S lim_ratio(int limiter, const S &u0, const S &g0, const S &g1, const S &g2, const S &x,
                                       const S &e2, const double cf[3]) {
  const S dM = g0 * cf[0] + g1 * cf[1] + g2 * cf[2];
  if (limiter == 3) {
    const double small = 1.e-12;
    const S dU = x - u0;
    S mm;
    if (dU * dM < 0.) mm = S(0.);
    else if (dU > 0.) mm = smin(dU, dM);
    else mm = smax(dU, dM);
    const double sU = (double)((mm > 0.) - (mm < 0.)), sG = (double)((dM > 0.) - (dM < 0.));
    return (mm + sU * small) / (dM + sG * small);
  }
  if (limiter == 1) {
    const S dP = x - u0;
    const S num = dP * dP + e2 + 2. * dM * dP;
    const S den = dP * dP + 2. * dM * dM + dM * dP + e2;
    return num / den;
  }
  return (x - u0) / dM;
}

// Cell stage (with the limiter adjoint).  Outputs the cell's own state and
// gradient adjoints; the contribution to the neighbour holding a limiter's
// extreme goes to Wface (one slot per variable, face and side, so no two
// threads write one slot) and the eps^2 adjoints to per-block partial sums.
template <bool VISCOUS>
__global__ void __launch_bounds__(128) k_cell_adj(DevCase cs, DevMesh m, const double *__restrict__ W,
                                                  const double *__restrict__ G, const double *__restrict__ Lm,
                                                  const unsigned long long *__restrict__ ext, const double *__restrict__ FA,
                                                  double *__restrict__ Wcell, double *__restrict__ Gb,
                                                  double *__restrict__ Wface, double *__restrict__ e2part) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int nc = m.nc, nt = m.nt, nf = m.nf;
  double e2b[5] = {0., 0., 0., 0., 0.};
  if (c < nc) {
    const double xc[3] = {m.c_x[c], m.c_x[nt + c], m.c_x[2 * nt + c]};
    double wb[5] = {0., 0., 0., 0., 0.}, lb[5] = {0., 0., 0., 0., 0.}, gb[15];
    double g[15], lm[5];
    for (int i = 0; i < 15; ++i) { gb[i] = 0.; g[i] = G[i * nc + c]; }
    for (int v = 0; v < 5; ++v) lm[v] = Lm[v * nc + c];
    const int f0 = m.cf_index[c], f1 = m.cf_index[c + 1];
    for (int j = f0; j < f1; ++j) {
      const int e = m.cf_list[j];
      const bool parent = e >= 0;
      const int f = parent ? e : ~e;
      const int q = parent ? U_QL : U_QR, cc = parent ? U_CL : U_CR, gg = parent ? U_GPA : U_GNB;
      const double d[3] = {m.f_x[f] - xc[0], m.f_x[nf + f] - xc[1], m.f_x[2 * nf + f] - xc[2]};
      for (int v = 0; v < 5; ++v) {
        const double qb = FA[(size_t)(q + v) * nf + f];
        wb[v] += qb + FA[(size_t)(cc + v) * nf + f];
        if (qb != 0.) {
          const double dot = d[0] * g[3 * v] + d[1] * g[3 * v + 1] + d[2] * g[3 * v + 2];
          lb[v] += qb * dot;
          for (int i = 0; i < 3; ++i) gb[3 * v + i] += qb * lm[v] * d[i];
        }
      }
      if (VISCOUS)
        for (int r = 0; r < 12; ++r) gb[3 + r] += FA[(size_t)(gg + r) * nf + f];
    }
    // limiter adjoint: phi_v = min over faces of the ratio; the derivative
    // follows the face that attained the minimum
    if (cs.order != 1 && cs.limiter > 0) {
      double u0[5], umax[5], umin[5];
      int amax[5], amin[5], amaxf[5], aminf[5];
      for (int v = 0; v < 5; ++v) {
        u0[v] = W[v * nt + c]; umax[v] = umin[v] = u0[v]; amax[v] = amin[v] = c; amaxf[v] = aminf[v] = -1;
      }
      if (cs.limiter != 3) {
        for (int j = f0; j < f1; ++j) {
          const int e = m.cf_list[j];
          const int f = e >= 0 ? e : ~e;
          const int o = e >= 0 ? m.f_neighbor[f] : m.f_parent[f];
          for (int v = 0; v < 5; ++v) {
            const double x = W[v * nt + o];
            if (umax[v] < x) { umax[v] = x; amax[v] = o; amaxf[v] = f; }
            if (x < umin[v]) { umin[v] = x; amin[v] = o; aminf[v] = f; }
          }
        }
      }
      double e2[5] = {0., 0., 0., 0., 0.};
      if (cs.limiter == 1) {
        // eps^2 as in k_grad_limiter (find_min_max with its index quirks)
        const double pmax = okey_inv(ext[0]), pmin = okey_inv(ext[1]);
        const double T0 = W[4 * nt + 0], wl = W[3 * nt + nc - 1];
        double qmax[5], qmin[5];
        qmax[0] = pmax; qmin[0] = pmin;
        qmax[1] = okey_inv(ext[2]); qmin[1] = okey_inv(ext[3]);
        qmax[2] = okey_inv(ext[4]); qmin[2] = okey_inv(ext[5]);
        double q4M = T0, q4m = T0;
        if (nc > 1) {
          const double a = okey_inv(ext[6]), bb = okey_inv(ext[7]);
          if (T0 < a) q4M = a;
          if (bb < T0) q4m = bb;
        }
        qmax[3] = q4M; if (q4M < wl) qmax[3] = wl;
        qmin[3] = q4m; if (wl < q4m) qmin[3] = wl;
        qmax[4] = T0; if (T0 < pmax) qmax[4] = pmax;
        qmin[4] = T0; if (pmin < T0) qmin[4] = pmin;
        for (int v = 0; v < 5; ++v) {
          const double ee = 1.e-6 * cs.K * (fabs(qmax[v] - qmin[v]) / cs.Lref);
          e2[v] = ee * ee;
        }
      }
      for (int v = 0; v < 5; ++v) {
        if (lb[v] == 0.) continue;
        // forward search for the face attaining the minimum (same rounded
        // operations and comparisons as k_grad_limiter)
        double phi = 1.;
        int best = -1, bx = c, bf = -1;
        double bcf[3] = {0., 0., 0.};
        for (int j = f0; j < f1; ++j) {
          const int e = m.cf_list[j];
          const int f = e >= 0 ? e : ~e;
          const double cf[3] = {sub_rn(m.f_x[f], xc[0]), sub_rn(m.f_x[nf + f], xc[1]), sub_rn(m.f_x[2 * nf + f], xc[2])};
          const double dM = add_rn(add_rn(mul_rn(g[3 * v], cf[0]), mul_rn(g[3 * v + 1], cf[1])), mul_rn(g[3 * v + 2], cf[2]));
          double r;
          int xcell, xface = f;
          if (cs.limiter == 3) {
            const int o = e >= 0 ? m.f_neighbor[f] : m.f_parent[f];
            const double dU = sub_rn(W[v * nt + o], u0[v]);
            double mm;
            if (dU * dM < 0.) mm = 0.;
            else if (dU > 0.) mm = (dM < dU) ? dM : dU;
            else mm = (dU < dM) ? dM : dU;
            const double sU = (double)((mm > 0.) - (mm < 0.)), sG = (double)((dM > 0.) - (dM < 0.));
            r = div_rn(add_rn(mm, sU * 1.e-12), add_rn(dM, sG * 1.e-12));
            xcell = o;
          } else if (cs.limiter == 1) {
            if (dM == 0.) continue;
            double dP;
            if (dM > 0.) { dP = sub_rn(umax[v], u0[v]); xcell = amax[v]; xface = amaxf[v]; }
            else { dP = sub_rn(umin[v], u0[v]); xcell = amin[v]; xface = aminf[v]; }
            const double dP2 = mul_rn(dP, dP), dM2 = mul_rn(dM, dM);
            const double num = add_rn(add_rn(dP2, e2[v]), mul_rn(mul_rn(2., dM), dP));
            const double den = add_rn(add_rn(add_rn(dP2, mul_rn(2., dM2)), mul_rn(dM, dP)), e2[v]);
            r = div_rn(num, den);
          } else {
            if (dM == 0.) { r = 1.; xcell = -1; }
            else if (dM > 0.) { r = div_rn(sub_rn(umax[v], u0[v]), dM); xcell = amax[v]; xface = amaxf[v]; }
            else { r = div_rn(sub_rn(umin[v], u0[v]), dM); xcell = amin[v]; xface = aminf[v]; }
          }
          if (r < phi) { phi = r; best = j; bx = xcell; bf = xface; bcf[0] = cf[0]; bcf[1] = cf[1]; bcf[2] = cf[2]; }
        }
        if (best < 0 || bx < 0) continue;
        const double s = lb[v];
        if (bx >= nc) {
          // the extreme / neighbour is this cell's own ghost, a function of
          // the cell's state (first-order BC): differentiate through it with
          // lanes p,u,v,w,T of the cell, g0..g2, eps^2 so that terms which
          // cancel exactly (a mirrored ghost) cancel in the tangent too
          typedef DN<9> D9;
          const double n[3] = {m.f_n[bf], m.f_n[nf + bf], m.f_n[2 * nf + bf]};
          FState<D9> Lc, Rg;
          Lc.p = D9(W[c]); Lc.V[0] = D9(W[nt + c]); Lc.V[1] = D9(W[2 * nt + c]); Lc.V[2] = D9(W[3 * nt + c]);
          Lc.T = D9(W[4 * nt + c]);
          Lc.p.d[0] = 1.; Lc.V[0].d[1] = 1.; Lc.V[1].d[2] = 1.; Lc.V[2].d[3] = 1.; Lc.T.d[4] = 1.;
          Lc.pc = Lc.p; Lc.Tc = Lc.T; Lc.Vc[0] = Lc.V[0]; Lc.Vc[1] = Lc.V[1]; Lc.Vc[2] = Lc.V[2];
          Lc.rho = eos_rho(cs, Lc.p, Lc.T);
          finish(cs, Lc, n);
          Rg.rho = D9(0.);
          apply_bc(cs, cs.bc[m.f_bc[bf]], Lc, Rg, n, (int *)nullptr);
          const D9 gst[5] = {Rg.p, Rg.V[0], Rg.V[1], Rg.V[2], Rg.T};
          const D9 cst[5] = {Lc.p, Lc.V[0], Lc.V[1], Lc.V[2], Lc.T};
          D9 b1(g[3 * v]), b2(g[3 * v + 1]), b3(g[3 * v + 2]), b5(e2[v]);
          b1.d[5] = 1.; b2.d[6] = 1.; b3.d[7] = 1.; b5.d[8] = 1.;
          const D9 r = lim_ratio<D9>(cs.limiter, cst[v], b1, b2, b3, gst[v], b5, bcf);
          for (int k = 0; k < 5; ++k) wb[k] += s * r.d[k];
          gb[3 * v] += s * r.d[5]; gb[3 * v + 1] += s * r.d[6]; gb[3 * v + 2] += s * r.d[7];
          e2b[v] += s * r.d[8];
          continue;
        }
        // lanes: u0, g0, g1, g2, x, e2
        typedef DN<6> D6;
        D6 a0(u0[v]), a1(g[3 * v]), a2(g[3 * v + 1]), a3(g[3 * v + 2]), a4(W[v * nt + bx]), a5(e2[v]);
        a0.d[0] = 1.; a1.d[1] = 1.; a2.d[2] = 1.; a3.d[3] = 1.; a5.d[5] = 1.;
        // when the cell itself holds the extreme, x and u0 are one variable:
        // one lane, so x - u0 has an exactly zero tangent (separate lanes
        // would cancel ~1/dM terms in floating point)
        a4.d[bx == c ? 0 : 4] = 1.;
        const D6 r = lim_ratio<D6>(cs.limiter, a0, a1, a2, a3, a4, a5, bcf);
        wb[v] += s * r.d[0];
        gb[3 * v] += s * r.d[1]; gb[3 * v + 1] += s * r.d[2]; gb[3 * v + 2] += s * r.d[3];
        // the extreme sits across face bf: this cell's contribution to it,
        // kept per (variable, face, side) and gathered in face order later
        if (bx != c) Wface[((size_t)v * 2 + (m.f_parent[bf] == c ? 0 : 1)) * nf + bf] = s * r.d[4];
        e2b[v] += s * r.d[5];
      }
    }
    for (int v = 0; v < 5; ++v) Wcell[v * nc + c] = wb[v];
    for (int i = 0; i < 15; ++i) Gb[i * nc + c] = gb[i];
  }
  // per-block partial sums of the eps^2 adjoints
  __shared__ double sh[5][4];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int v = 0; v < 5; ++v) {
    double t = e2b[v];
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (lane == 0) sh[v][wid] = t;
  }
  __syncthreads();
  if (threadIdx.x < 5) {
    double t = 0.;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += sh[threadIdx.x][k];
    e2part[(size_t)blockIdx.x * 5 + threadIdx.x] = t;
  }
}

// eps^2 adjoints -> the cells that supplied the global extrema.
__global__ void k_e2_adj(DevCase cs, DevMesh m, const double *__restrict__ W, const unsigned long long *__restrict__ ext,
                         const int *__restrict__ argx, const double *__restrict__ e2part, int nparts,
                         double *__restrict__ Wlim) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const int nc = m.nc, nt = m.nt;
  double e2b[5] = {0., 0., 0., 0., 0.};
  for (int k = 0; k < nparts; ++k)
    for (int v = 0; v < 5; ++v) e2b[v] += e2part[(size_t)k * 5 + v];
  // ten sources: slots 0..7 (cells argx[slot]) and T of cell 0, w of cell nc-1
  typedef DN<10> D10;
  const int var_of[8] = {0, 0, 1, 1, 2, 2, 0, 0};
  D10 src[10];
  for (int k = 0; k < 8; ++k) { src[k] = D10(okey_inv(ext[k])); src[k].d[k] = 1.; }
  src[8] = D10(W[4 * nt + 0]); src[8].d[8] = 1.;
  src[9] = D10(W[3 * nt + nc - 1]); src[9].d[9] = 1.;
  const D10 &pmax = src[0], &pmin = src[1], &T0 = src[8], &wl = src[9];
  D10 qmax[5], qmin[5];
  qmax[0] = pmax; qmin[0] = pmin;
  qmax[1] = src[2]; qmin[1] = src[3];
  qmax[2] = src[4]; qmin[2] = src[5];
  D10 q4M = T0, q4m = T0;
  if (nc > 1) {
    if (T0 < src[6]) q4M = src[6];
    if (src[7] < T0) q4m = src[7];
  }
  qmax[3] = q4M; if (q4M < wl) qmax[3] = wl;
  qmin[3] = q4m; if (wl < q4m) qmin[3] = wl;
  qmax[4] = T0; if (T0 < pmax) qmax[4] = pmax;
  qmin[4] = T0; if (pmin < T0) qmin[4] = pmin;
  double sb[10];
  for (int k = 0; k < 10; ++k) sb[k] = 0.;
  for (int v = 0; v < 5; ++v) {
    const D10 ee = 1.e-6 * cs.K * (fabs(qmax[v] - qmin[v]) / cs.Lref);
    const D10 e2 = ee * ee;
    for (int k = 0; k < 10; ++k) sb[k] += e2b[v] * e2.d[k];
  }
  for (int k = 0; k < 8; ++k) {
    const int cell = argx[k];
    if (sb[k] != 0. && cell >= 0 && cell < nc) Wlim[(size_t)var_of[k] * nt + cell] += sb[k];
  }
  if (sb[8] != 0.) Wlim[(size_t)4 * nt + 0] += sb[8];
  if (sb[9] != 0.) Wlim[(size_t)3 * nt + nc - 1] += sb[9];
}

// Gradient stage: Wgrad_k = sum over cells c whose stencil holds k of
// w_ck . Gbar_c (transposed stencil, ascending c), for NV variables (the
// flow's 5, or k and omega).
template <int NV>
__global__ void k_grad_adj(DevMesh m, const int *__restrict__ tr_index, const int *__restrict__ tr_cell,
                           const int *__restrict__ tr_entry, const double *__restrict__ Gb, double *__restrict__ Wgrad) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int nc = m.nc, nt = m.nt;
  if (k >= nt) return;
  double acc[NV];
  for (int v = 0; v < NV; ++v) acc[v] = 0.;
  const double xk[3] = {m.c_x[k], m.c_x[nt + k], m.c_x[2 * nt + k]};
  for (int j = tr_index[k]; j < tr_index[k + 1]; ++j) {
    const int c = tr_cell[j];
    double wt[3];
    if (m.st_w) {
      // stored map weights (curvilinear cases): entry tr_entry[j] of c's map
      const size_t e = (size_t)tr_entry[j];
      wt[0] = m.st_w[3 * e]; wt[1] = m.st_w[3 * e + 1]; wt[2] = m.st_w[3 * e + 2];
    } else if (c == k) {
      wt[0] = m.st_self[c]; wt[1] = m.st_self[nc + c]; wt[2] = m.st_self[2 * nc + c];
    } else {
      const double d0 = xk[0] - m.c_x[c], d1 = xk[1] - m.c_x[nt + c], d2 = xk[2] - m.c_x[2 * nt + c];
      const double w = (d0 * d0 + d1 * d1 + d2 * d2) / m.st_cof[6 * nc + c];
      const double C00 = m.st_cof[c], C01 = m.st_cof[nc + c], C02 = m.st_cof[2 * nc + c];
      const double C11 = m.st_cof[3 * nc + c], C12 = m.st_cof[4 * nc + c], C22 = m.st_cof[5 * nc + c];
      wt[0] = w * (d0 * C00 + d1 * C01 + d2 * C02);
      wt[1] = w * (d0 * C01 + d1 * C11 + d2 * C12);
      wt[2] = w * (d0 * C02 + d1 * C12 + d2 * C22);
    }
    for (int v = 0; v < NV; ++v)
      acc[v] += wt[0] * Gb[(3 * v) * nc + c] + wt[1] * Gb[(3 * v + 1) * nc + c] + wt[2] * Gb[(3 * v + 2) * nc + c];
  }
  for (int v = 0; v < NV; ++v) Wgrad[(size_t)v * nt + k] = acc[v];
}

// Ghost stage: ghost t (boundary face bface[t]) is the first-order BC state
// of its parent; GA[.][t] = (d ghost / d W_parent)^T gbar.
// Wx ([5][nb], may be null): further adjoints of the ghost states (the
// k-omega terms of a turbulent case).
__global__ void k_ghost_adj(DevCase cs, DevMesh m, const double *__restrict__ W, const double *__restrict__ FA,
                            const double *__restrict__ Wgrad, const double *__restrict__ Wlim,
                            const double *__restrict__ Wx, double *__restrict__ GA) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= m.nb) return;
  const int nt = m.nt, nf = m.nf, nc = m.nc;
  const int f = m.bface[t], pa = m.f_parent[f], b = m.f_bc[f], g = nc + t;
  double gbar[5];
  bool any = false;
  for (int v = 0; v < 5; ++v) {
    gbar[v] = FA[(size_t)(U_CR + v) * nf + f] + Wgrad[(size_t)v * nt + g] + Wlim[(size_t)v * nt + g];
    if (Wx) gbar[v] += Wx[(size_t)v * m.nb + t];
    any = any || gbar[v] != 0.;
  }
  double out[5] = {0., 0., 0., 0., 0.};
  if (any) {
    const double n[3] = {m.f_n[f], m.f_n[nf + f], m.f_n[2 * nf + f]};
    typedef DN<5> D5;
    FState<D5> L, R;
    L.p = D5(W[pa]); L.V[0] = D5(W[nt + pa]); L.V[1] = D5(W[2 * nt + pa]); L.V[2] = D5(W[3 * nt + pa]); L.T = D5(W[4 * nt + pa]);
    L.p.d[0] = 1.; L.V[0].d[1] = 1.; L.V[1].d[2] = 1.; L.V[2].d[3] = 1.; L.T.d[4] = 1.;
    L.pc = L.p; L.Tc = L.T; L.Vc[0] = L.V[0]; L.Vc[1] = L.V[1]; L.Vc[2] = L.V[2];
    L.rho = eos_rho(cs, L.p, L.T);
    finish(cs, L, n);
    R.rho = D5(0.);
    apply_bc(cs, cs.bc[b], L, R, n, (int *)nullptr);
    const D5 gv[5] = {R.p, R.V[0], R.V[1], R.V[2], R.T};
    for (int k = 0; k < 5; ++k) {
      double s = 0.;
      for (int v = 0; v < 5; ++v) s += gbar[v] * gv[v].d[k];
      out[k] = s;
    }
  }
  for (int k = 0; k < 5; ++k) GA[(size_t)k * m.nb + t] = out[k];
}

// Final gather per cell: Wbar = cell + gradient + limiter-neighbour terms +
// its ghosts' parent terms (ascending face order).
template <bool AOS>
__global__ void k_final_adj(DevMesh m, const double *__restrict__ Wcell, const double *__restrict__ Wgrad,
                            const double *__restrict__ Wlim, const double *__restrict__ GA, double *__restrict__ out) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int nc = m.nc, nt = m.nt, nf = m.nf;
  if (c >= nc) return;
  double r[5];
  for (int v = 0; v < 5; ++v) r[v] = Wcell[v * nc + c] + Wgrad[(size_t)v * nt + c] + Wlim[(size_t)v * nt + c];
  for (int j = m.cf_index[c]; j < m.cf_index[c + 1]; ++j) {
    const int e = m.cf_list[j];
    if (e < 0) continue;
    if (m.f_bc[e] < 0) continue;
    const int t = m.f_neighbor[e] - nc;
    for (int v = 0; v < 5; ++v) r[v] += GA[(size_t)v * m.nb + t];
  }
  (void)nf;
  for (int v = 0; v < 5; ++v) {
    if (AOS) out[5 * c + v] = r[v];
    else out[v * nc + c] = r[v];
  }
}

// Sum of -D[1..3] over the faces of the selected regions: per-block partials.
__global__ void k_loads(DevMesh m, const double *__restrict__ D, unsigned int mask, double *__restrict__ part) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  double s[3] = {0., 0., 0.};
  if (f < m.nf) {
    const int b = m.f_bc[f];
    if (b >= 0 && ((mask >> b) & 1u))
      for (int i = 0; i < 3; ++i) s[i] = -D[(size_t)(1 + i) * m.nf + f];
  }
  __shared__ double sh[3][8];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int i = 0; i < 3; ++i) {
    double t = s[i];
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (lane == 0) sh[i][wid] = t;
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    double t = 0.;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += sh[threadIdx.x][k];
    part[(size_t)blockIdx.x * 3 + threadIdx.x] = t;
  }
}

__global__ void k_rearm(unsigned long long *ext, int *argx) {
  const int t = threadIdx.x;
  if (t < 8) {
    ext[t] = (t & 1) ? ~0ull : 0ull;
    argx[t] = 0x7F7F7F7F;
  }
}

// ---- k-omega stages of a turbulent case (reverse of the k-omega half of
// the coupled evaluation: eddy viscosity, its face values, the k / omega
// gradients, face fluxes, gather and sources; kw.cuh).

// local inputs of a k-omega face flux (kw_face_flux)
enum { KW_TPA = 0, KW_TNB = 1, KW_KL = 2, KW_OL = 3, KW_KR = 4, KW_OR = 5, KW_GPA = 6, KW_GNB = 12, KW_MUTF = 18, KW_MDOT = 19,
       KW_WL = 20, KW_N = 21 };

// Face stage: RFA[i][f] = sum_v DKbar_v dDK_v/du_i with DKbar from RKbar by
// the gather's transpose (+ for the parent, - for the neighbour).
__global__ void __launch_bounds__(128) k_kw_face_adj(DevCase cs, DevMesh m, const double *__restrict__ W,
                                                     const double *__restrict__ K, const double *__restrict__ GK,
                                                     const double *__restrict__ mutf, const double *__restrict__ mdot,
                                                     const double *__restrict__ wl, const double *__restrict__ RKb,
                                                     double *__restrict__ RFA) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  const int nf = m.nf, nc = m.nc, nt = m.nt;
  if (f >= nf) return;
  const int pa = m.f_parent[f], nb = m.f_neighbor[f], b = m.f_bc[f];
  const double db0 = RKb[pa] - (b < 0 ? RKb[nb] : 0.), db1 = RKb[nc + pa] - (b < 0 ? RKb[nc + nb] : 0.);
  double ub[KW_N];
  for (int i = 0; i < KW_N; ++i) ub[i] = 0.;
  if (db0 != 0. || db1 != 0.) {
    double u[KW_N];
    u[KW_TPA] = W[4 * nt + pa]; u[KW_TNB] = W[4 * nt + nb];
    u[KW_KL] = K[pa]; u[KW_OL] = K[nt + pa]; u[KW_KR] = K[nb]; u[KW_OR] = K[nt + nb];
    for (int i = 0; i < 6; ++i) {
      u[KW_GPA + i] = GK[i * nc + pa];
      u[KW_GNB + i] = b < 0 ? GK[i * nc + nb] : 0.;
    }
    u[KW_MUTF] = mutf[f]; u[KW_MDOT] = mdot[f]; u[KW_WL] = wl[f];
    int act[KW_N], na = 0;
    const bool tfix = b >= 0 && cs.bc[b].T_fixed;
    for (int i = 0; i < KW_N; ++i) {
      if (tfix && (i == KW_TPA || i == KW_TNB)) continue;
      if (b >= 0 && i >= KW_GNB && i < KW_GNB + 6) continue;
      act[na++] = i;
    }
    for (int k0 = 0; k0 < na; k0 += kLanes) {
      Seeds in;
      in.u = u;
      for (int l = 0; l < kLanes; ++l) in.chunk[l] = (k0 + l < na) ? act[k0 + l] : -1;
      DA gpa[6], gnb[6];
      for (int i = 0; i < 6; ++i) { gpa[i] = in(KW_GPA + i); gnb[i] = in(KW_GNB + i); }
      DA d0, d1;
      kw_face_flux<DA>(cs, m, f, b, pa, nb, in(KW_TPA), in(KW_TNB), in(KW_KL), in(KW_OL), in(KW_KR), in(KW_OR), gpa, gnb,
                       in(KW_MUTF), in(KW_MDOT), in(KW_WL), d0, d1);
      for (int l = 0; l < kLanes; ++l)
        if (in.chunk[l] >= 0) ub[in.chunk[l]] = db0 * d0.d[l] + db1 * d1.d[l];
    }
  }
  for (int i = 0; i < KW_N; ++i) RFA[(size_t)i * nf + f] = ub[i];
}

// (p, T, k, omega) adjoints of mu_t = kw_mut(p, T, k, omega), scaled by mb
__device__ __forceinline__ void kw_mut_adj(const DevCase &cs, double p, double T, double k, double om, double ratio,
                                           double mb, double out[4]) {
  typedef DN<4> D4;
  D4 a(p), t(T), kk(k), o(om);
  a.d[0] = 1.; t.d[1] = 1.; kk.d[2] = 1.; o.d[3] = 1.;
  const D4 r = kw_mut<D4>(cs, a, t, kk, o, ratio);
  for (int i = 0; i < 4; ++i) out[i] = mb * r.d[i];
}

// Cell stage: per cell, the k-omega faces' adjoints of its T, k, omega and
// k / omega gradient (its side of each face, ascending face order), the face
// eddy viscosities' adjoints (the face value is the weighted average of the
// two cells' unless the BC fixes it), the sources' adjoints (velocity
// gradient rows into Gb, p and T into Wcell) and the cell eddy viscosity's
// (into p, T, k, omega).  Kcell: k, omega adjoints ([2][nc]); GKb: the k /
// omega gradients' ([6][nc]).
__global__ void __launch_bounds__(128) k_kw_cell_adj(DevCase cs, DevMesh m, const double *__restrict__ W,
                                                     const double *__restrict__ K, const double *__restrict__ G,
                                                     const double *__restrict__ mut, const double *__restrict__ vol,
                                                     const double *__restrict__ RKb, const double *__restrict__ RFA,
                                                     const double *__restrict__ FA, double ratio,
                                                     double *__restrict__ Wcell, double *__restrict__ Gb,
                                                     double *__restrict__ Kcell, double *__restrict__ GKb) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int nc = m.nc, nt = m.nt, nf = m.nf;
  if (c >= nc) return;
  double pb = 0., tb = 0., kb[2] = {0., 0.}, gkb[6] = {0., 0., 0., 0., 0., 0.}, mb = 0.;
  for (int j = m.cf_index[c]; j < m.cf_index[c + 1]; ++j) {
    const int e = m.cf_list[j];
    const bool parent = e >= 0;
    const int f = parent ? e : ~e;
    tb += RFA[(size_t)(parent ? KW_TPA : KW_TNB) * nf + f];
    kb[0] += RFA[(size_t)(parent ? KW_KL : KW_KR) * nf + f];
    kb[1] += RFA[(size_t)(parent ? KW_OL : KW_OR) * nf + f];
    for (int i = 0; i < 6; ++i) gkb[i] += RFA[(size_t)((parent ? KW_GPA : KW_GNB) + i) * nf + f];
    const int b = m.f_bc[f];
    if (!(b >= 0 && cs.bc[b].mut_fixed))
      mb += (parent ? m.f_w[f] : m.f_w[nf + f]) * (RFA[(size_t)KW_MUTF * nf + f] + FA[(size_t)U_MUT * nf + f]);
  }
  // sources: inputs g9 (0..8), p, T, k, omega, mu_t (9..13)
  const double sb0 = RKb[c] * vol[c], sb1 = RKb[nc + c] * vol[c];
  double sbar[14];
  for (int i = 0; i < 14; ++i) sbar[i] = 0.;
  if (sb0 != 0. || sb1 != 0.) {
    double u[14];
    for (int i = 0; i < 9; ++i) u[i] = G[(3 + i) * nc + c];
    u[9] = W[c]; u[10] = W[4 * nt + c]; u[11] = K[c]; u[12] = K[nt + c]; u[13] = mut[c];
    for (int k0 = 0; k0 < 14; k0 += kLanes) {
      Seeds in;
      in.u = u;
      for (int l = 0; l < kLanes; ++l) in.chunk[l] = (k0 + l < 14) ? k0 + l : -1;
      DA g9[9];
      for (int i = 0; i < 9; ++i) g9[i] = in(i);
      DA s0, s1;
      kw_source<DA>(cs, g9, in(9), in(10), in(11), in(12), in(13), s0, s1);
      for (int l = 0; l < kLanes; ++l)
        if (in.chunk[l] >= 0) sbar[in.chunk[l]] = sb0 * s0.d[l] + sb1 * s1.d[l];
    }
  }
  pb += sbar[9]; tb += sbar[10]; kb[0] += sbar[11]; kb[1] += sbar[12]; mb += sbar[13];
  if (mb != 0.) {
    double a[4];
    kw_mut_adj(cs, W[c], W[4 * nt + c], K[c], K[nt + c], ratio, mb, a);
    pb += a[0]; tb += a[1]; kb[0] += a[2]; kb[1] += a[3];
  }
  for (int i = 0; i < 9; ++i) Gb[(size_t)(3 + i) * nc + c] += sbar[i];
  Wcell[c] += pb;
  Wcell[(size_t)4 * nc + c] += tb;
  Kcell[c] = kb[0];
  Kcell[nc + c] = kb[1];
  for (int i = 0; i < 6; ++i) GKb[(size_t)i * nc + c] = gkb[i];
}

// Ghost stage: ghost t's T, k, omega adjoints from its boundary face's
// k-omega flux and the k / omega gradients' stencils (Kgrad), and its eddy
// viscosity's (the face value's neighbour weight, unless the BC fixes it).
// Wx: the ghost's p, T adjoints for the flow's ghost stage ([5][nb]); KGA:
// the ghost's k, omega adjoints for its parent ([2][nb]; zero where the BC
// fixes k and omega).
__global__ void k_kw_ghost_adj(DevCase cs, DevMesh m, const double *__restrict__ W, const double *__restrict__ K,
                               const double *__restrict__ RFA, const double *__restrict__ FA,
                               const double *__restrict__ Kgrad, double ratio, double *__restrict__ Wx,
                               double *__restrict__ KGA) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int nb = m.nb, nc = m.nc, nt = m.nt, nf = m.nf;
  if (t >= nb) return;
  const int f = m.bface[t], b = m.f_bc[f], g = nc + t;
  double tb = RFA[(size_t)KW_TNB * nf + f], pb = 0.;
  double kb0 = RFA[(size_t)KW_KR * nf + f] + Kgrad[g], kb1 = RFA[(size_t)KW_OR * nf + f] + Kgrad[nt + g];
  const double mb = cs.bc[b].mut_fixed ? 0. : m.f_w[nf + f] * (RFA[(size_t)KW_MUTF * nf + f] + FA[(size_t)U_MUT * nf + f]);
  if (mb != 0.) {
    double a[4];
    kw_mut_adj(cs, W[g], W[4 * nt + g], K[g], K[nt + g], ratio, mb, a);
    pb += a[0]; tb += a[1]; kb0 += a[2]; kb1 += a[3];
  }
  for (int v = 0; v < 5; ++v) Wx[(size_t)v * nb + t] = v == 0 ? pb : (v == 4 ? tb : 0.);
  const bool fixed = cs.bc[b].kw_fixed;
  KGA[t] = fixed ? 0. : kb0;
  KGA[nb + t] = fixed ? 0. : kb1;
}

// Kbar per cell (AoS [nc][2]): its own terms, its k / omega stencil terms
// and its ghosts' (boundary faces in ascending order).
__global__ void k_kw_final_adj(DevMesh m, const double *__restrict__ Kcell, const double *__restrict__ Kgrad,
                               const double *__restrict__ KGA, double *__restrict__ out) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int nc = m.nc, nt = m.nt;
  if (c >= nc) return;
  double r[2] = {Kcell[c] + Kgrad[c], Kcell[nc + c] + Kgrad[nt + c]};
  for (int j = m.cf_index[c]; j < m.cf_index[c + 1]; ++j) {
    const int e = m.cf_list[j];
    if (e < 0 || m.f_bc[e] < 0) continue;
    const int t = m.f_neighbor[e] - nc;
    r[0] += KGA[t];
    r[1] += KGA[m.nb + t];
  }
  out[2 * c] = r[0];
  out[2 * c + 1] = r[1];
}

// k-omega staging (SoA [2][nc]) of a turbulent case's RKbar
__global__ void k_aos2_to_soa(const double *__restrict__ in, double *__restrict__ out, int nc) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  out[c] = in[2 * c];
  out[nc + c] = in[2 * c + 1];
}

struct AdjBufs {
  DBuf<double> FA, Wcell, Gb, Wlim, Wgrad, GA, e2part, Rb, out;
  // turbulent cases: k-omega face adjoints, cell / gradient / ghost terms, staging
  DBuf<double> RFA, Kcell, GKb, Kgrad, Wx, KGA, RKb, Kin, Kout;
  bool kw_ready = false;
  DBuf<double> Wface, SC;  // per-face-side limiter contributions; outlet faces' stale-density adjoints
  DBuf<int> tr_index, tr_cell, tr_entry, tgt;
  bool ready = false;
};

}  // namespace

// Adjoint buffers live with the context (allocated on first use).
struct AdjointState {
  AdjBufs b;
};

void adjoint_free(fcfd_ctx *x) {
  delete x->adj;
  x->adj = nullptr;
}

static AdjBufs &adj_bufs(fcfd_ctx *x) {
  if (!x->adj) x->adj = new AdjointState();
  AdjBufs &a = x->adj->b;
  if (a.ready) return a;
  const DevMesh &m = x->dm;
  const fcfd_mesh &h = *x->mesh;
  const int nc = m.nc, nt = m.nt;
  // transposed LSQ stencil over all nt cells (ascending c per column)
  std::vector<int> cnt(nt + 1, 0);
  for (int c = 0; c < nc; ++c)
    for (int j = h.st_index[c]; j < h.st_index[c + 1]; ++j) cnt[h.st_keys[j] + 1]++;
  for (int k = 0; k < nt; ++k) cnt[k + 1] += cnt[k];
  std::vector<int> cells(cnt[nt]), entries(cnt[nt]);
  std::vector<int> fill(cnt.begin(), cnt.end() - 1);
  for (int c = 0; c < nc; ++c)
    for (int j = h.st_index[c]; j < h.st_index[c + 1]; ++j) {
      entries[fill[h.st_keys[j]]] = j;
      cells[fill[h.st_keys[j]]++] = c;
    }
  a.tr_index.upload(cnt);
  if (!cells.empty()) { a.tr_cell.upload(cells); a.tr_entry.upload(entries); }
  a.FA.alloc((size_t)U_N * m.nf);
  a.Wcell.alloc(5 * (size_t)nc);
  a.Gb.alloc(15 * (size_t)nc);
  a.Wlim.alloc(5 * (size_t)nt);
  a.Wface.alloc(10 * (size_t)m.nf);
  a.SC.alloc((size_t)U_N * std::max(m.n_outlet, 1));
  a.tgt.alloc((size_t)std::max(m.n_outlet, 1));
  a.Wgrad.alloc(5 * (size_t)nt);
  a.GA.alloc(5 * (size_t)std::max(m.nb, 1));
  a.e2part.alloc(5 * (size_t)((nc + 127) / 128 + 1));
  a.Rb.alloc(5 * (size_t)nc);
  a.out.alloc(5 * (size_t)nc);
  a.ready = true;
  return a;
}

static void kw_adj_bufs(fcfd_ctx *x, AdjBufs &a) {
  if (a.kw_ready) return;
  const DevMesh &m = x->dm;
  const int nc = m.nc, nt = m.nt, nb = std::max(m.nb, 1);
  a.RFA.alloc((size_t)KW_N * m.nf);
  a.Kcell.alloc(2 * (size_t)nc); a.GKb.alloc(6 * (size_t)nc); a.Kgrad.alloc(2 * (size_t)nt);
  a.Wx.alloc(5 * (size_t)nb); a.KGA.alloc(2 * (size_t)nb);
  a.RKb.alloc(2 * (size_t)nc); a.Kin.alloc(2 * (size_t)nc); a.Kout.alloc(2 * (size_t)nc);
  a.kw_ready = true;
}

// The k-omega half of a turbulent case's reverse sweep: the forward
// evaluation's arrays, the seed RKbar (SoA [2][nc]) and the output Kbar (AoS
// [nc][2], device).
struct KwAdj {
  RansFwd fw;
  const double *RKb;
  double *Kout;
};

// Reverse sweep for seed Rbar (SoA [5][nc], may be null) and/or the load
// seed (mask, dir); the forward state must already be in x->p64.W (interior).
// kw: a turbulent case's k-omega seed and output (the forward evaluation of
// rans_eval_for_adjoint already run), else null.
static void run_adjoint(fcfd_ctx *x, const double *Rbar_soa, unsigned int mask, const double dir[3], double *out, bool aos,
                        const KwAdj *kw = nullptr) {
  const DevMesh &m = x->dm;
  cudaStream_t s = x->stream;
  const int tb = 256;
  Pipe<double> &P = x->p64;
  AdjBufs &a = adj_bufs(x);
  // forward: ghosts + extrema, first attaining cells, gradient + limiter, stale density
  const bool need_ext = x->cs.limiter == 1 && x->cs.order != 1;
  const int ng = (m.nb + tb - 1) / tb + (need_ext ? kExtremaBlocks : 0);
  if (ng > 0) k_ghost_minmax<double><<<ng, tb, 0, s>>>(x->cs, m, P.W.p, need_ext ? x->ext.p : nullptr, x->err.p);
  if (need_ext) k_argext<double><<<(m.nc + tb - 1) / tb, tb, 0, s>>>(m, P.W.p, x->ext.p, x->argx.p);
  launch_grad_limiter<double>(x->cs, m, P.W.p, x->ext.p, nullptr, P.G.p, P.Lm.p, s);
  if (m.n_outlet > 0)
    k_outlet_rho<double><<<(m.n_outlet + 127) / 128, 128, 0, s>>>(x->cs, m, P.W.p, P.G.p, P.Lm.p, P.stale.p);
  // reverse
  const int gf = (m.nf + 127) / 128, gc = (m.nc + 127) / 128;
  const double *mutf = nullptr, *mdotb = nullptr, *wlb = nullptr;
  if (kw) {
    // k-omega faces first: their mdot and weightL adjoints seed the flow's faces
    k_kw_face_adj<<<gf, 128, 0, s>>>(x->cs, m, P.W.p, kw->fw.K, kw->fw.GK, kw->fw.mutf, kw->fw.mdot, kw->fw.wl, kw->RKb,
                                     a.RFA.p);
    mutf = kw->fw.mutf;
    mdotb = a.RFA.p + (size_t)KW_MDOT * m.nf;
    wlb = a.RFA.p + (size_t)KW_WL * m.nf;
  }
  if (x->viscous)
    FCFD_BY_FLUX(x->cs.flux, k_face_adj<true, FX><<<gf, 128, 0, s>>>(x->cs, m, P.W.p, P.G.p, P.Lm.p, P.stale.p, Rbar_soa, mask, dir[0], dir[1], dir[2], mutf, mdotb, wlb, a.FA.p));
  else
    FCFD_BY_FLUX(x->cs.flux, k_face_adj<false, FX><<<gf, 128, 0, s>>>(x->cs, m, P.W.p, P.G.p, P.Lm.p, P.stale.p, Rbar_soa, mask, dir[0], dir[1], dir[2], mutf, mdotb, wlb, a.FA.p));
  if (m.n_outlet > 0) {
    const int go = (m.n_outlet + 127) / 128;
    CK(cudaMemsetAsync(a.SC.p, 0, sizeof(double) * U_N * (size_t)m.n_outlet, s));
    CK(cudaMemsetAsync(a.tgt.p, 0xFF, sizeof(int) * (size_t)m.n_outlet, s));
    if (x->viscous) FCFD_BY_FLUX(x->cs.flux, k_stale_adj<true, FX><<<go, 128, 0, s>>>(x->cs, m, P.W.p, P.G.p, P.Lm.p, P.stale.p, mutf, a.FA.p, a.SC.p, a.tgt.p));
    else FCFD_BY_FLUX(x->cs.flux, k_stale_adj<false, FX><<<go, 128, 0, s>>>(x->cs, m, P.W.p, P.G.p, P.Lm.p, P.stale.p, mutf, a.FA.p, a.SC.p, a.tgt.p));
    k_stale_apply<<<go, 128, 0, s>>>(m.n_outlet, m.nf, a.SC.p, a.tgt.p, a.FA.p);
  }
  CK(cudaMemsetAsync(a.Wlim.p, 0, sizeof(double) * 5 * (size_t)m.nt, s));
  CK(cudaMemsetAsync(a.Wface.p, 0, sizeof(double) * 10 * (size_t)m.nf, s));
  if (x->viscous)
    k_cell_adj<true><<<gc, 128, 0, s>>>(x->cs, m, P.W.p, P.G.p, P.Lm.p, x->ext.p, a.FA.p, a.Wcell.p, a.Gb.p, a.Wface.p, a.e2part.p);
  else
    k_cell_adj<false><<<gc, 128, 0, s>>>(x->cs, m, P.W.p, P.G.p, P.Lm.p, x->ext.p, a.FA.p, a.Wcell.p, a.Gb.p, a.Wface.p, a.e2part.p);
  if (kw)
    k_kw_cell_adj<<<gc, 128, 0, s>>>(x->cs, m, P.W.p, kw->fw.K, P.G.p, kw->fw.mut, kw->fw.vol, kw->RKb, a.RFA.p, a.FA.p,
                                     kw->fw.ratio, a.Wcell.p, a.Gb.p, a.Kcell.p, a.GKb.p);
  k_wlim_gather<<<(5 * m.nc + 255) / 256, 256, 0, s>>>(m, a.Wface.p, a.Wlim.p);
  if (need_ext) k_e2_adj<<<1, 32, 0, s>>>(x->cs, m, P.W.p, x->ext.p, x->argx.p, a.e2part.p, gc, a.Wlim.p);
  k_grad_adj<5><<<(m.nt + 127) / 128, 128, 0, s>>>(m, a.tr_index.p, a.tr_cell.p, a.tr_entry.p, a.Gb.p, a.Wgrad.p);
  if (kw) {
    k_grad_adj<2><<<(m.nt + 127) / 128, 128, 0, s>>>(m, a.tr_index.p, a.tr_cell.p, a.tr_entry.p, a.GKb.p, a.Kgrad.p);
    if (m.nb > 0)
      k_kw_ghost_adj<<<(m.nb + 127) / 128, 128, 0, s>>>(x->cs, m, P.W.p, kw->fw.K, a.RFA.p, a.FA.p, a.Kgrad.p, kw->fw.ratio,
                                                        a.Wx.p, a.KGA.p);
  }
  if (m.nb > 0)
    k_ghost_adj<<<(m.nb + 127) / 128, 128, 0, s>>>(x->cs, m, P.W.p, a.FA.p, a.Wgrad.p, a.Wlim.p, kw ? a.Wx.p : nullptr, a.GA.p);
  if (aos) k_final_adj<true><<<(m.nc + tb - 1) / tb, tb, 0, s>>>(m, a.Wcell.p, a.Wgrad.p, a.Wlim.p, a.GA.p, out);
  else k_final_adj<false><<<(m.nc + tb - 1) / tb, tb, 0, s>>>(m, a.Wcell.p, a.Wgrad.p, a.Wlim.p, a.GA.p, out);
  if (kw) k_kw_final_adj<<<(m.nc + tb - 1) / tb, tb, 0, s>>>(m, a.Kcell.p, a.Kgrad.p, a.KGA.p, kw->Kout);
  k_rearm<<<1, 32, 0, s>>>(x->ext.p, x->argx.p);
  CK(cudaGetLastError());
}

}  // namespace fcfd

using namespace fcfd;

extern "C" {

int fcfd_vjp(fcfd_ctx *x, const double *W, const double *Rbar, double *Wbar, int flags) {
  try {
    if (!x || !W || !Rbar || !Wbar) throw Error(FCFD_ERR_INPUT, "null argument");
    if (x->green_gauss) throw Error(FCFD_ERR_UNSUPPORTED, "the adjoint covers least-squares gradients only");
    CK(cudaSetDevice(x->device));
    const DevMesh &m = x->dm;
    cudaStream_t s = x->stream;
    const bool dev = flags & FCFD_DEVICE_PTRS;
    const size_t n = 5 * (size_t)m.nc;
    AdjBufs &a = adj_bufs(x);
    const double *w = W, *rb = Rbar;
    if (!dev) {
      CK(cudaMemcpyAsync(x->Win.p, W, sizeof(double) * n, cudaMemcpyHostToDevice, s));
      CK(cudaMemcpyAsync(a.out.p, Rbar, sizeof(double) * n, cudaMemcpyHostToDevice, s));
      w = x->Win.p;
      rb = a.out.p;
    }
    const int tb = 256;
    k_aos_to_soa<double><<<(m.nc + tb - 1) / tb, tb, 0, s>>>(w, x->p64.W.p, m.nc, m.nt);
    k_aos_to_soa<double><<<(m.nc + tb - 1) / tb, tb, 0, s>>>(rb, a.Rb.p, m.nc, m.nc);
    const double dir[3] = {0., 0., 0.};
    double *out = dev ? Wbar : a.out.p;
    run_adjoint(x, a.Rb.p, 0u, dir, out, true);
    if (!dev) CK(cudaMemcpyAsync(Wbar, a.out.p, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    check_err(x);
  } catch (const Error &e) {
    set_last_error(e.what());
    return e.code;
  } catch (const std::exception &e) {
    set_last_error(e.what());
    return FCFD_ERR_INPUT;
  }
  return FCFD_OK;
}

// (Wbar, Kbar) = (d(R, RK)/d(W, K))^T (Rbar, RKbar) for a turbulent case:
// the flow adjoint above with the k-omega terms reversed as well.
int fcfd_rans_vjp(fcfd_ctx *x, const double *W, const double *K, const double *Rbar, const double *RKbar, double *Wbar,
                  double *Kbar, int flags) {
  try {
    if (!x || !W || !K || !Rbar || !RKbar || !Wbar || !Kbar) throw Error(FCFD_ERR_INPUT, "null argument");
    if (!x->rans) throw Error(FCFD_ERR_INPUT, "the case has no turbulence model");
    CK(cudaSetDevice(x->device));
    const DevMesh &m = x->dm;
    cudaStream_t s = x->stream;
    const bool dev = flags & FCFD_DEVICE_PTRS;
    const size_t n = 5 * (size_t)m.nc, nk = 2 * (size_t)m.nc;
    AdjBufs &a = adj_bufs(x);
    kw_adj_bufs(x, a);
    const double *w = W, *k = K, *rb = Rbar, *rkb = RKbar;
    if (!dev) {
      CK(cudaMemcpyAsync(x->Win.p, W, sizeof(double) * n, cudaMemcpyHostToDevice, s));
      CK(cudaMemcpyAsync(a.Kin.p, K, sizeof(double) * nk, cudaMemcpyHostToDevice, s));
      CK(cudaMemcpyAsync(a.out.p, Rbar, sizeof(double) * n, cudaMemcpyHostToDevice, s));
      CK(cudaMemcpyAsync(a.Kout.p, RKbar, sizeof(double) * nk, cudaMemcpyHostToDevice, s));
      w = x->Win.p; k = a.Kin.p; rb = a.out.p; rkb = a.Kout.p;
    }
    const int tb = 256;
    KwAdj kw;
    rans_eval_for_adjoint(x, w, k, kw.fw);
    k_aos_to_soa<double><<<(m.nc + tb - 1) / tb, tb, 0, s>>>(rb, a.Rb.p, m.nc, m.nc);
    k_aos2_to_soa<<<(m.nc + tb - 1) / tb, tb, 0, s>>>(rkb, a.RKb.p, m.nc);
    kw.RKb = a.RKb.p;
    kw.Kout = dev ? Kbar : a.Kout.p;
    const double dir[3] = {0., 0., 0.};
    double *out = dev ? Wbar : a.out.p;
    run_adjoint(x, a.Rb.p, 0u, dir, out, true, &kw);
    if (!dev) {
      CK(cudaMemcpyAsync(Wbar, a.out.p, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
      CK(cudaMemcpyAsync(Kbar, a.Kout.p, sizeof(double) * nk, cudaMemcpyDeviceToHost, s));
    }
    CK(cudaStreamSynchronize(s));
    check_err(x);
  } catch (const Error &e) {
    set_last_error(e.what());
    return e.code;
  } catch (const std::exception &e) {
    set_last_error(e.what());
    return FCFD_ERR_INPUT;
  }
  return FCFD_OK;
}

int fcfd_drag(fcfd_ctx *x, const double *W, uint32_t bc_mask, const double *dir, double *force, double *dJdW, int flags) {
  try {
    if (!x || !W || !dir || !force) throw Error(FCFD_ERR_INPUT, "null argument");
    if (dJdW && x->green_gauss) throw Error(FCFD_ERR_UNSUPPORTED, "the adjoint covers least-squares gradients only");
    CK(cudaSetDevice(x->device));
    const DevMesh &m = x->dm;
    cudaStream_t s = x->stream;
    const bool dev = flags & FCFD_DEVICE_PTRS;
    const size_t n = 5 * (size_t)m.nc;
    AdjBufs &a = adj_bufs(x);
    const double *w = W;
    if (!dev) {
      CK(cudaMemcpyAsync(x->Win.p, W, sizeof(double) * n, cudaMemcpyHostToDevice, s));
      w = x->Win.p;
    }
    const int tb = 256;
    k_aos_to_soa<double><<<(m.nc + tb - 1) / tb, tb, 0, s>>>(w, x->p64.W.p, m.nc, m.nt);
    launch_chain<double>(x, x->p64, x->p64.R.p, false, nullptr, nullptr);
    const int nblk = (m.nf + tb - 1) / tb;
    DBuf<double> part;
    part.alloc(3 * (size_t)nblk);
    k_loads<<<nblk, tb, 0, s>>>(m, x->p64.D.p, bc_mask, part.p);
    std::vector<double> hp(3 * (size_t)nblk);
    CK(cudaMemcpyAsync(hp.data(), part.p, sizeof(double) * hp.size(), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    check_err(x);
    double F[3] = {0., 0., 0.};
    for (int k = 0; k < nblk; ++k)
      for (int i = 0; i < 3; ++i) F[i] += hp[3 * (size_t)k + i];
    for (int i = 0; i < 3; ++i) force[i] = F[i];
    if (dJdW) {
      double *out = dev ? dJdW : a.out.p;
      run_adjoint(x, nullptr, bc_mask, dir, out, true);
      if (!dev) CK(cudaMemcpyAsync(dJdW, a.out.p, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
      CK(cudaStreamSynchronize(s));
    }
  } catch (const Error &e) {
    set_last_error(e.what());
    return e.code;
  } catch (const std::exception &e) {
    set_last_error(e.what());
    return FCFD_ERR_INPUT;
  }
  return FCFD_OK;
}

}  // extern "C"
