// Matrix-free Newton-Krylov solve of R(W) = 0 on the device.
//
// Pseudo-transient continuation as in the reference's implicit step
// (NavierStokes::solve, ns.cc:104-118):  (V P/dt - dR/dW) dW = R(W),
// W <- W + dW, with P the conservative-to-primitive Jacobian of
// NavierStokes::cons2prim (ns_time_terms.cc:26-56) and dt the local time step
// of update_time_step (time_step.cc:143-224).  The reference assembles a
// finite-difference Jacobian and hands it to PETSc FGMRES; here the Jacobian is
// never stored:
//   * Jacobian-vector products come either from a finite difference of the
//     FP64 residual ("plain") or from the dual-number tangent kernels
//     (fcfd_jvp's chain; "jvp"), optionally with an FP32 Krylov basis;
//   * the preconditioner is block Jacobi: per cell the 5x5 block
//     V P/dt - sum_faces dD_f/dW_c of the first-order face Jacobians (the
//     reference's get_jacobians perturbs the reconstructed face states the same
//     way), computed with 5-lane dual numbers and inverted in place;
//   * GMRES(m) with right preconditioning; Gram-Schmidt (classical, applied
//     twice) accumulates every dot product in FP64 with a fixed reduction
//     order, so a solve is bit-reproducible.
#include <sys/stat.h>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <string>
#include <type_traits>
#include <vector>

#include "ctx.hpp"
#include "dn.cuh"

namespace fcfd {

typedef DN<5> D5;

struct RowScale {
  double s[5];  // per-equation weight of the GMRES norm
};

// Per-Newton-step scalars of the Krylov iteration.  The kernels read them from
// device memory, so an iteration captured once as a CUDA graph stays valid
// when they change from one Newton step to the next.
struct IterConsts {
  RowScale rs;     // GMRES row weights
  RowScale winv;   // 1 / per-variable reference magnitudes
  RowScale one;    // unit weights
  double eps_num;  // finite-difference step numerator
};

// ------------------------------------------------------------------ face Jacobians
__device__ __forceinline__ void seed(const FState<double> &s, FState<D5> &o, const DevCase &cs, const double n[3]) {
  // perturbations of state_perturb (ns_assemble_linear_system.cc:417-458):
  // p moves the face pressure only; u,v,w move V and V_center; T moves T and T_center
  o.p = D5(s.p); o.p.d[0] = 1.;
  o.pc = D5(s.pc);
  for (int i = 0; i < 3; ++i) { o.V[i] = D5(s.V[i]); o.V[i].d[1 + i] = 1.; o.Vc[i] = D5(s.Vc[i]); o.Vc[i].d[1 + i] = 1.; }
  o.T = D5(s.T); o.T.d[4] = 1.;
  o.Tc = D5(s.Tc); o.Tc.d[4] = 1.;
  o.rho = eos_rho(cs, o.p, o.T);
  finish(cs, o, n);
}
__device__ __forceinline__ void lift(const FState<double> &s, FState<D5> &o) {
  o.p = D5(s.p); o.T = D5(s.T); o.rho = D5(s.rho); o.a = D5(s.a); o.H = D5(s.H); o.Vn = D5(s.Vn);
  o.pc = D5(s.pc); o.Tc = D5(s.Tc);
  for (int i = 0; i < 3; ++i) { o.V[i] = D5(s.V[i]); o.Vc[i] = D5(s.Vc[i]); }
}

// Per face: JL = dD/dW_left and (interior faces) JR = dD/dW_right, [25][nf],
// entry (i,k) = d D_i / d W_k at index (5i+k)*nf + f.
template <bool VISCOUS, int FX>
__global__ void __launch_bounds__(128) k_face_jac(DevCase cs, DevMesh m, const double *__restrict__ W, const double *__restrict__ G,
                                                  const double *__restrict__ Lm, const double *__restrict__ stale,
                                                  double *__restrict__ JL, double *__restrict__ JR,
                                                  const double *__restrict__ mutf = nullptr) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  const int nf = m.nf;
  if (f >= nf) return;
  const int pa = m.f_parent[f], nb = m.f_neighbor[f], b = m.f_bc[f];
  const double n[3] = {m.f_n[f], m.f_n[nf + f], m.f_n[2 * nf + f]};
  const double A = m.f_area[f];
  FState<double> L, R;
  face_states(cs, m, f, n, b, pa, nb, W, G, Lm, const_cast<double *>(stale), L, R, (int *)nullptr);
  FState<D5> Ld, Rd;
  D5 D[5], wl;
  const GlobalGrad<double> gs{G, m.nc, pa, nb};
  seed(L, Ld, cs, n);
  if (b < 0) {
    lift(R, Rd);
  } else {
    Rd.pc = D5(R.pc); Rd.Tc = D5(R.Tc); Rd.rho = D5(0.);
    for (int i = 0; i < 3; ++i) Rd.Vc[i] = D5(R.Vc[i]);
    if (!apply_bc(cs, cs.bc[b], Ld, Rd, n, (int *)nullptr)) Rd.rho = D5(R.rho);
    finish(cs, Rd, n);
  }
  face_D<D5, GlobalGrad<double>, VISCOUS, FX>(cs, m, f, n, A, b, pa, nb, Ld, Rd, gs, mutf, D, wl);
#pragma unroll
  for (int i = 0; i < 5; ++i)
#pragma unroll
    for (int k = 0; k < 5; ++k) JL[(5 * i + k) * nf + f] = D[i].d[k];
  if (b < 0) {
    lift(L, Ld);
    seed(R, Rd, cs, n);
    face_D<D5, GlobalGrad<double>, VISCOUS, FX>(cs, m, f, n, A, b, pa, nb, Ld, Rd, gs, mutf, D, wl);
#pragma unroll
    for (int i = 0; i < 5; ++i)
#pragma unroll
      for (int k = 0; k < 5; ++k) JR[(5 * i + k) * nf + f] = D[i].d[k];
  }
}

// cons2prim (ns_time_terms.cc:26-56): P[i][k] = d(rho, rho u, rho v, rho w, rho E)_i / d(p,u,v,w,T)_k
__device__ __forceinline__ void cons2prim(const DevCase &cs, double p, double u, double v, double w, double T, double P[25]) {
  const double pressure = p + cs.Pref, temperature = T + cs.Tref;
  const double rho = pressure / (cs.R * temperature);
  const double drho_dT = -1. * rho / temperature, drho_dp = rho / pressure;
  const double c_p = cs.Cp;
  const double H = c_p * temperature + 0.5 * (u * u + v * v + w * w);
  for (int i = 0; i < 25; ++i) P[i] = 0.;
  P[0] = drho_dp; P[4] = drho_dT;
  P[5] = drho_dp * u; P[6] = rho; P[9] = drho_dT * u;
  P[10] = drho_dp * v; P[12] = rho; P[14] = drho_dT * v;
  P[15] = drho_dp * w; P[18] = rho; P[19] = drho_dT * w;
  P[20] = drho_dp * H - 1.; P[21] = rho * u; P[22] = rho * v; P[23] = rho * w; P[24] = drho_dT * H + rho * c_p;
}

// Diagonal block of cell c of the implicit operator: V P/dt - J_cc, J_cc the
// cell's own first-order face Jacobians in ascending face order (minus the
// parent side's JL, plus the neighbour side's JR).
__device__ __forceinline__ void diag_block(const DevCase &cs, const DevMesh &m, const double *__restrict__ Wn,
                                           const double *__restrict__ vol, const double *__restrict__ dt,
                                           const double *__restrict__ JL, const double *__restrict__ JR, int c,
                                           double B[25]) {
  const int nc = m.nc, nf = m.nf;
  cons2prim(cs, Wn[c], Wn[nc + c], Wn[2 * nc + c], Wn[3 * nc + c], Wn[4 * nc + c], B);
  const double s = vol[c] / dt[c];
#pragma unroll
  for (int i = 0; i < 25; ++i) B[i] *= s;
  for (int j = m.cf_index[c]; j < m.cf_index[c + 1]; ++j) {
    const int e = m.cf_list[j];
    if (e >= 0) {
#pragma unroll
      for (int i = 0; i < 25; ++i) B[i] -= JL[i * nf + e];
    } else {
      const int f = ~e;
#pragma unroll
      for (int i = 0; i < 25; ++i) B[i] += JR[i * nf + f];
    }
  }
}

// The assembled diagonal blocks themselves, [nc][25] (fcfd_diag_blocks).
__global__ void k_diag_blocks(DevCase cs, DevMesh m, const double *__restrict__ Wn, const double *__restrict__ vol,
                              const double *__restrict__ dt, const double *__restrict__ JL, const double *__restrict__ JR,
                              double *__restrict__ out) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= m.nc) return;
  double B[25];
  diag_block(cs, m, Wn, vol, dt, JL, JR, c, B);
#pragma unroll
  for (int i = 0; i < 25; ++i) out[25 * (size_t)c + i] = B[i];
}

// Time-term blocks V P/dt per cell ([nc][25], row = equation, column =
// primitive variable): NavierStokes::time_terms (ns_time_terms.cc:107-186)
// with cons2prim (26-56).
__global__ void k_time_blocks(DevCase cs, int nc, const double *__restrict__ Wn, const double *__restrict__ vol,
                              const double *__restrict__ dt, double *__restrict__ out) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  double P[25];
  cons2prim(cs, Wn[c], Wn[nc + c], Wn[2 * nc + c], Wn[3 * nc + c], Wn[4 * nc + c], P);
  const double sc = vol[c] / dt[c];
#pragma unroll
  for (int i = 0; i < 25; ++i) out[25 * (size_t)c + i] = sc * P[i];
}

// Block assembly + inversion (Gauss-Jordan, partial pivoting): Minv_c = (V P/dt - J_cc)^-1
__global__ void k_block_jacobi(DevCase cs, DevMesh m, const double *__restrict__ Wn, const double *__restrict__ vol,
                               const double *__restrict__ dt, const double *__restrict__ JL, const double *__restrict__ JR,
                               double *__restrict__ Minv, int *__restrict__ err, RowScale wref,
                               double *__restrict__ rowmag) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int nc = m.nc;
  if (c >= nc) return;
  double B[25];
  diag_block(cs, m, Wn, vol, dt, JL, JR, c, B);
  // magnitude of each equation's row for reference state changes: sum_k |B_ik| Wref_k
#pragma unroll
  for (int i = 0; i < 5; ++i) {
    double s = 0.;
#pragma unroll
    for (int k = 0; k < 5; ++k) s += ::fabs(B[5 * i + k]) * wref.s[k];
    rowmag[i * nc + c] = s;
  }
  double I[25];
#pragma unroll
  for (int i = 0; i < 25; ++i) I[i] = (i % 6 == 0) ? 1. : 0.;
  for (int col = 0; col < 5; ++col) {
    int piv = col;
    double best = ::fabs(B[5 * col + col]);
    for (int r = col + 1; r < 5; ++r)
      if (::fabs(B[5 * r + col]) > best) { best = ::fabs(B[5 * r + col]); piv = r; }
    if (!(best > 0.)) { atomicOr(err, 4); best = 1.; }
    if (piv != col)
      for (int k = 0; k < 5; ++k) {
        double t = B[5 * col + k]; B[5 * col + k] = B[5 * piv + k]; B[5 * piv + k] = t;
        t = I[5 * col + k]; I[5 * col + k] = I[5 * piv + k]; I[5 * piv + k] = t;
      }
    const double inv = 1. / B[5 * col + col];
    for (int k = 0; k < 5; ++k) { B[5 * col + k] *= inv; I[5 * col + k] *= inv; }
    for (int r = 0; r < 5; ++r) {
      if (r == col) continue;
      const double fct = B[5 * r + col];
      for (int k = 0; k < 5; ++k) { B[5 * r + k] -= fct * B[5 * col + k]; I[5 * r + k] -= fct * I[5 * col + k]; }
    }
  }
#pragma unroll
  for (int i = 0; i < 25; ++i) Minv[i * nc + c] = I[i];
}

// Block ILU(0) of the first-order operator A = B + O in the multicolour
// order (colours ascending, cells of one colour never face neighbours):
// modified diagonal blocks Dt_i = B_i - sum over face neighbours j of an
// earlier colour of A_ij Dt_j^-1 A_ji, with A_ij = -JR_f, A_ji = +JL_f when i
// is face f's parent and A_ij = +JL_f, A_ji = -JR_f when it is its
// neighbour (the signs of k_jacobi_sweep).  This is the incomplete LU with
// no fill when no three cells are pairwise face neighbours (hexahedra,
// prisms: every other product falls outside the sparsity pattern); around
// tetrahedral edges the fill between two neighbours of j is dropped (the
// diagonal form of ILU(0)).  One launch per colour, in colour order; writes
// Dt_i^-1 ([25][nc], by cell) for the cells of colour `col`.
__global__ void k_ilu_diag(DevCase cs, DevMesh m, const double *__restrict__ Wn, const double *__restrict__ vol,
                           const double *__restrict__ dt, const double *__restrict__ JL, const double *__restrict__ JR,
                           int deg, int cnt, int col, const int *__restrict__ cells, const int *__restrict__ nbr,
                           const int *__restrict__ src, const int *__restrict__ colour, double *__restrict__ MinvT,
                           int *__restrict__ err) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= cnt) return;
  const int nc = m.nc, nf = m.nf;
  const int c = cells[i];
  double B[25];
  diag_block(cs, m, Wn, vol, dt, JL, JR, c, B);
  for (int sl = 0; sl < deg; ++sl) {
    const int o = nbr[(size_t)sl * cnt + i];
    if (o < 0 || colour[o] >= col) continue;
    const int e = src[(size_t)sl * cnt + i];
    const int f = e >= 0 ? e : ~e;
    const double *Jij = e >= 0 ? JR : JL, *Jji = e >= 0 ? JL : JR;
    const double sij = e >= 0 ? -1. : 1., sji = -sij;
    // T = Dt_o^-1 A_oc (5x5), then B -= A_co T
    double T[25];
#pragma unroll
    for (int r = 0; r < 5; ++r)
#pragma unroll
      for (int q = 0; q < 5; ++q) {
        double a = 0.;
#pragma unroll
        for (int k = 0; k < 5; ++k) a += MinvT[(size_t)(5 * r + k) * nc + o] * (sji * Jji[(size_t)(5 * k + q) * nf + f]);
        T[5 * r + q] = a;
      }
#pragma unroll
    for (int r = 0; r < 5; ++r)
#pragma unroll
      for (int q = 0; q < 5; ++q) {
        double a = 0.;
#pragma unroll
        for (int k = 0; k < 5; ++k) a += (sij * Jij[(size_t)(5 * r + k) * nf + f]) * T[5 * k + q];
        B[5 * r + q] -= a;
      }
  }
  double I[25];
#pragma unroll
  for (int q = 0; q < 25; ++q) I[q] = (q % 6 == 0) ? 1. : 0.;
  for (int cc = 0; cc < 5; ++cc) {
    int piv = cc;
    double best = ::fabs(B[5 * cc + cc]);
    for (int r = cc + 1; r < 5; ++r)
      if (::fabs(B[5 * r + cc]) > best) { best = ::fabs(B[5 * r + cc]); piv = r; }
    if (!(best > 0.)) { atomicOr(err, 4); best = 1.; }
    if (piv != cc)
      for (int k = 0; k < 5; ++k) {
        double t = B[5 * cc + k]; B[5 * cc + k] = B[5 * piv + k]; B[5 * piv + k] = t;
        t = I[5 * cc + k]; I[5 * cc + k] = I[5 * piv + k]; I[5 * piv + k] = t;
      }
    const double inv = 1. / B[5 * cc + cc];
    for (int k = 0; k < 5; ++k) { B[5 * cc + k] *= inv; I[5 * cc + k] *= inv; }
    for (int r = 0; r < 5; ++r) {
      if (r == cc) continue;
      const double fct = B[5 * r + cc];
      for (int k = 0; k < 5; ++k) { B[5 * r + k] -= fct * B[5 * cc + k]; I[5 * r + k] -= fct * I[5 * cc + k]; }
    }
  }
#pragma unroll
  for (int q = 0; q < 25; ++q) MinvT[(size_t)q * nc + c] = I[q];
}

// z = Minv x (per-cell 5x5), vectors [5][nc] of type T
// z = Minv (D^-1 x): right preconditioner of the row-scaled system D A
template <class T>
__global__ void k_precond(int nc, const double *__restrict__ Minv, const T *__restrict__ x, T *__restrict__ z,
                          const RowScale *__restrict__ rs) {
  pdl_wait();
  pdl_trigger();
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  double xv[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) xv[k] = double(x[k * nc + c]) / rs->s[k];
#pragma unroll
  for (int i = 0; i < 5; ++i) {
    double s = 0.;
#pragma unroll
    for (int k = 0; k < 5; ++k) s += Minv[(5 * i + k) * nc + c] * xv[k];
    z[i * nc + c] = T(s);
  }
}

// r = D^-1 v rounded to the preconditioner's type P, y = Minv r: the start of
// the Gauss-Seidel preconditioner in one pass
// (bar: the persistent Gauss-Seidel kernel's barrier counter, zeroed here, or null)
template <class T, class P>
__global__ void k_precond_split(int nc, const double *__restrict__ Minv, const T *__restrict__ v,
                                const RowScale *__restrict__ rs, P *__restrict__ r, P *__restrict__ y,
                                unsigned *bar = nullptr) {
  pdl_wait();
  pdl_trigger();
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (bar && c == 0) bar[0] = 0u;
  if (c >= nc) return;
  double xv[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    const P rk = P(double(v[k * nc + c]) / rs->s[k]);
    r[k * nc + c] = rk;
    xv[k] = double(rk);
  }
#pragma unroll
  for (int i = 0; i < 5; ++i) {
    double s = 0.;
#pragma unroll
    for (int k = 0; k < 5; ++k) s += Minv[(5 * i + k) * nc + c] * xv[k];
    y[i * nc + c] = P(s);
  }
}

// One block-Jacobi sweep on the first-order operator A1 = B + O:
// y_out = Binv (r - O y_in), with (O y)_c = -sum_{f: c parent} JR_f y_nb + sum_{f: c neighbour} JL_f y_parent.
template <class T>
__global__ void k_jacobi_sweep(DevMesh m, const double *__restrict__ Minv, const double *__restrict__ JL,
                               const double *__restrict__ JR, const double *__restrict__ r, const double *__restrict__ yin,
                               double *__restrict__ yout) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int nc = m.nc, nf = m.nf;
  if (c >= nc) return;
  double t[5];
#pragma unroll
  for (int i = 0; i < 5; ++i) t[i] = r[i * nc + c];
  for (int j = m.cf_index[c]; j < m.cf_index[c + 1]; ++j) {
    const int e = m.cf_list[j];
    const int f = e >= 0 ? e : ~e;
    if (m.f_bc[f] >= 0) continue;  // boundary faces have no off-diagonal block
    const int o = e >= 0 ? m.f_neighbor[f] : m.f_parent[f];
    const double *J = e >= 0 ? JR : JL;
    const double sg = e >= 0 ? 1. : -1.;  // r - O y
    double yo[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) yo[k] = yin[k * nc + o];
#pragma unroll
    for (int i = 0; i < 5; ++i) {
      double a = 0.;
#pragma unroll
      for (int k = 0; k < 5; ++k) a += J[(5 * i + k) * nf + f] * yo[k];
      t[i] += sg * a;
    }
  }
#pragma unroll
  for (int i = 0; i < 5; ++i) {
    double s = 0.;
#pragma unroll
    for (int k = 0; k < 5; ++k) s += Minv[(5 * i + k) * nc + c] * t[k];
    yout[i * nc + c] = s;
  }
}

// Pack one colour's couplings for the Gauss-Seidel kernel: the signed
// off-diagonal blocks (slot-major [deg][25][cnt]) and the inverse diagonal
// blocks ([25][cnt]), so that consecutive threads read consecutive words.
template <class P>
__global__ void k_pack_gs(int nc, int nf, int deg, int cnt, const int *__restrict__ cells, const int *__restrict__ nbr,
                          const int *__restrict__ src, const double *__restrict__ JL, const double *__restrict__ JR,
                          const double *__restrict__ Minv, P *__restrict__ OB, P *__restrict__ MinvP) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= cnt) return;
  const int c = cells[i];
#pragma unroll
  for (int q = 0; q < 25; ++q) MinvP[(size_t)q * cnt + i] = P(Minv[(size_t)q * nc + c]);
  for (int sl = 0; sl < deg; ++sl) {
    const int o = nbr[(size_t)sl * cnt + i], e = src[(size_t)sl * cnt + i];
    const int f = e >= 0 ? e : ~e;
    const double *J = e >= 0 ? JR : JL;
    const double sg = e >= 0 ? 1. : -1.;
#pragma unroll
    for (int q = 0; q < 25; ++q) OB[((size_t)sl * 25 + q) * cnt + i] = P(o >= 0 ? sg * J[(size_t)q * nf + f] : 0.);
  }
}

// Block Gauss-Seidel update of the cells of one colour, in place, from the
// packed couplings: y_c = Binv (r - O y)_c (no two cells of a colour share a
// face, so the cells update independently).
constexpr int kGsMaxDeg = 6;  // interior faces per cell of hexes, prisms, tetrahedra

// One thread per (cell, row): a block holds 32 cells of
// the colour and five warps, warp q taking row q of all 32 cells, so every
// load of the packed couplings ([deg][25][cnt], cells consecutive) is one
// contiguous 32-word row and no lane idles; the rows meet in shared memory
// for the diagonal solve.  (Eight lanes per cell with five active and the rows
// meeting through shuffles measured 14.5 / 8.4 us per FP64 / FP32 colour
// update on the 256x128 cylinder; this layout 9.4 / 7.7 us.)
template <class P>
__global__ void __launch_bounds__(160) k_gs_rows(int nc, int deg, int cnt, const int *__restrict__ cells,
                                                 const int *__restrict__ nbr, const P *__restrict__ OB,
                                                 const P *__restrict__ MinvP, const P *__restrict__ r, P *__restrict__ y) {
  // consecutive colour updates are programmatic dependent launches: wait for
  // the previous colour's writes, let the next colour's launch overlap this tail
  pdl_wait();
  pdl_trigger();
  const int i = blockIdx.x * 32 + threadIdx.x, q = threadIdx.y;
  __shared__ P ts[5][32];
  const bool act = i < cnt;
  int c = 0;
  P t = P(0.);
  if (act) {
    c = cells[i];
    t = r[q * nc + c];
    if (deg <= kGsMaxDeg) {
      int o[kGsMaxDeg];
#pragma unroll
      for (int sl = 0; sl < kGsMaxDeg; ++sl) o[sl] = sl < deg ? nbr[(size_t)sl * cnt + i] : -1;
      P yv[kGsMaxDeg][5];
#pragma unroll
      for (int sl = 0; sl < kGsMaxDeg; ++sl)
#pragma unroll
        for (int k = 0; k < 5; ++k) yv[sl][k] = o[sl] >= 0 ? y[k * nc + o[sl]] : P(0.);
#pragma unroll
      for (int sl = 0; sl < kGsMaxDeg; ++sl) {
        if (o[sl] < 0) continue;
        const P *B = OB + ((size_t)sl * 25 + 5 * q) * cnt + i;
        P a = P(0.);
#pragma unroll
        for (int k = 0; k < 5; ++k) a += B[(size_t)k * cnt] * yv[sl][k];
        t += a;
      }
    } else {
      for (int sl = 0; sl < deg; ++sl) {
        const int o = nbr[(size_t)sl * cnt + i];
        if (o < 0) continue;
        const P *B = OB + ((size_t)sl * 25 + 5 * q) * cnt + i;
        P a = P(0.);
#pragma unroll
        for (int k = 0; k < 5; ++k) a += B[(size_t)k * cnt] * y[k * nc + o];
        t += a;
      }
    }
  }
  ts[q][threadIdx.x] = t;
  __syncthreads();
  if (act) {
    P v = P(0.);
#pragma unroll
    for (int k = 0; k < 5; ++k) v += MinvP[(size_t)(5 * q + k) * cnt + i] * ts[k][threadIdx.x];
    y[q * nc + c] = v;
  }
}

// ---- all colour updates of one preconditioner application in one launch
//
// The per-colour launches above leave a 16k-cell colour update latency-bound
// (a few microseconds of work per launch, most of it the launch ramp and the
// dependent index -> neighbour loads).  Here one cooperative grid runs every
// colour update of the symmetric sweeps in turn, with a grid-wide barrier
// between updates: block b takes the b-th chunk of each colour's cells, so
// with STAGE its couplings, inverse diagonal blocks, neighbour lists and
// right-hand side are read from HBM once per application into shared memory
// (they fit for FP32 couplings up to ~60k cells on 148 SMs) and every update
// reads them from there; only the neighbours' y crosses the barrier, through
// L2 (ld.global.cg).  The arithmetic per (cell, row) is k_gs_rows's, in the
// same order.  The barrier is an arrival counter that the preceding
// k_precond_split zeroes; a block that waits longer than kGsSpinLimit polls
// sets the timeout word and every later barrier of the launch stops waiting,
// so the launch always ends and the host reports FCFD_ERR_TIMEOUT.
constexpr int kGsZ = 4;                   // 32-cell groups per block (640 threads)
constexpr int kGsMaxCol = 32;             // colours of the greedy face-neighbour colouring
constexpr unsigned kGsSpinLimit = 1u << 22;  // polls of ~64 ns: > 0.25 s per barrier

struct GsPersistArgs {
  int nc, deg, ncol, nphase;
  const int *sched;   // [nphase] colour of each update
  const int *cells;   // cells by colour
  const int *nbr;     // [deg][cells of the colour] per colour
  unsigned *bar;      // [0] arrivals (zeroed before the launch), [1] timeout flag
  int cidx[kGsMaxCol + 1];  // colour offsets
  int soff[kGsMaxCol + 1];  // STAGE: offset of each colour's chunk in the staged arrays (prefix sums of chunk sizes)
};

__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned *p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// grid barrier number `k` (1-based) of the launch: every block arrives once.
// The block's writes are ordered before the arrival by __syncthreads and the
// release reduction (cumulative); the acquire load that sees every arrival
// orders the other blocks' writes before this block's later reads.
__device__ __forceinline__ void gs_grid_barrier(unsigned *bar, unsigned k) {
  __syncthreads();
  if (threadIdx.x == 0 && threadIdx.y == 0 && threadIdx.z == 0) {
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(bar), "r"(1u) : "memory");
    const unsigned target = k * gridDim.x;
    if (!ld_acquire_gpu(&bar[1])) {
      unsigned it = 0;
      while (ld_acquire_gpu(&bar[0]) < target) {
        if (++it > kGsSpinLimit) {
          atomicExch(&bar[1], 1u);
          break;
        }
        if (it > 256) __nanosleep(32);
      }
    }
  }
  __syncthreads();
}

template <class P, bool STAGE, int DMAX>
__global__ void __launch_bounds__(32 * 5 * kGsZ, 1) k_gs_persist(GsPersistArgs a, const P *__restrict__ OB,
                                                                 const P *__restrict__ MinvP, const P *__restrict__ r,
                                                                 P *y) {
  extern __shared__ __align__(16) unsigned char gs_smem[];
  constexpr int NG = 32 * kGsZ;  // cells per pass
  const int lx = threadIdx.x, q = threadIdx.y, z = threadIdx.z;
  const int tid = lx + 32 * (q + 5 * z), nthr = 32 * 5 * kGsZ;
  const int nb = gridDim.x, b = blockIdx.x, nc = a.nc, deg = a.deg;
  P *ts = reinterpret_cast<P *>(gs_smem);  // [5][NG]
  // staged arrays (STAGE): per colour, this block's chunk at offset soff[col]
  // with stride ch = chunk size of the colour
  const int stot = a.soff[a.ncol];
  P *sOB = ts + 5 * NG;                       // [stot * deg * 25]
  P *sMi = sOB + (size_t)stot * deg * 25;     // [stot * 25]
  P *sR = sMi + (size_t)stot * 25;            // [stot * 5]
  int *sCell = reinterpret_cast<int *>(sR + (size_t)stot * 5);  // [stot]
  int *sNbr = sCell + stot;                   // [stot * deg]
  if constexpr (STAGE) {
    for (int col = 0; col < a.ncol; ++col) {
      const int base = a.cidx[col], cnt = a.cidx[col + 1] - base;
      const int ch = a.soff[col + 1] - a.soff[col];
      const int lo = b * ch, n = max(0, min(cnt, lo + ch) - lo);
      const int so = a.soff[col];
      for (int t = tid; t < n; t += nthr) {
        const int c = a.cells[base + lo + t];
        sCell[so + t] = c;
        for (int v = 0; v < 5; ++v) sR[(size_t)so * 5 + v * ch + t] = r[(size_t)v * nc + c];
      }
      for (int t = tid; t < n * deg; t += nthr) {
        const int sl = t / n, i = t - sl * n;
        sNbr[(size_t)so * deg + sl * ch + i] = a.nbr[(size_t)base * deg + (size_t)sl * cnt + lo + i];
      }
      for (int t = tid; t < n * deg * 25; t += nthr) {
        const int e = t / n, i = t - e * n;  // e = slot * 25 + entry
        sOB[(size_t)so * deg * 25 + (size_t)e * ch + i] = OB[(size_t)base * deg * 25 + (size_t)e * cnt + lo + i];
      }
      for (int t = tid; t < n * 25; t += nthr) {
        const int e = t / n, i = t - e * n;
        sMi[(size_t)so * 25 + (size_t)e * ch + i] = MinvP[(size_t)base * 25 + (size_t)e * cnt + lo + i];
      }
    }
    __syncthreads();
  }
  for (int ph = 0; ph < a.nphase; ++ph) {
    const int col = a.sched[ph];
    const int base = a.cidx[col], cnt = a.cidx[col + 1] - base;
    const int ch = STAGE ? a.soff[col + 1] - a.soff[col] : (cnt + nb - 1) / nb;
    const int lo = b * ch, hi = min(cnt, lo + ch);
    const int so = STAGE ? a.soff[col] : 0;
    for (int i0 = lo; i0 < hi; i0 += NG) {
      const int i = i0 + 32 * z + lx, li = i - lo;
      const bool act = i < hi;
      int c = 0;
      P t = P(0.);
      if (act) {
        if constexpr (STAGE) {
          c = sCell[so + li];
          t = sR[(size_t)so * 5 + q * ch + li];
        } else {
          c = a.cells[base + i];
          t = r[(size_t)q * nc + c];
        }
        int o[DMAX];
#pragma unroll
        for (int sl = 0; sl < DMAX; ++sl)
          o[sl] = sl < deg ? (STAGE ? sNbr[(size_t)so * deg + sl * ch + li] : a.nbr[(size_t)base * deg + (size_t)sl * cnt + i])
                           : -1;
        P yv[DMAX][5];
#pragma unroll
        for (int sl = 0; sl < DMAX; ++sl)
#pragma unroll
          for (int k = 0; k < 5; ++k) yv[sl][k] = o[sl] >= 0 ? __ldcg(y + (size_t)k * nc + o[sl]) : P(0.);
#pragma unroll
        for (int sl = 0; sl < DMAX; ++sl) {
          if (o[sl] < 0) continue;
          P acc = P(0.);
          if constexpr (STAGE) {
            const P *B = sOB + (size_t)so * deg * 25 + (size_t)(sl * 25 + 5 * q) * ch + li;
#pragma unroll
            for (int k = 0; k < 5; ++k) acc += B[(size_t)k * ch] * yv[sl][k];
          } else {
            const P *B = OB + (size_t)base * deg * 25 + ((size_t)sl * 25 + 5 * q) * cnt + i;
#pragma unroll
            for (int k = 0; k < 5; ++k) acc += B[(size_t)k * cnt] * yv[sl][k];
          }
          t += acc;
        }
      }
      ts[q * NG + 32 * z + lx] = t;
      __syncthreads();
      if (act) {
        P v = P(0.);
        if constexpr (STAGE) {
#pragma unroll
          for (int k = 0; k < 5; ++k) v += sMi[(size_t)so * 25 + (size_t)(5 * q + k) * ch + li] * ts[k * NG + 32 * z + lx];
        } else {
#pragma unroll
          for (int k = 0; k < 5; ++k) v += MinvP[(size_t)base * 25 + (size_t)(5 * q + k) * cnt + i] * ts[k * NG + 32 * z + lx];
        }
        y[(size_t)q * nc + c] = v;
      }
      __syncthreads();
    }
    if (ph + 1 < a.nphase) gs_grid_barrier(a.bar, (unsigned)(ph + 1));
  }
}

// copy a [5][nc] state into the residual chain's [5][nt] array (+ optional eps*dir)
// Finite-difference step eps = eps_num / |z| with |z|^2 read from the device
// (eps_num alone where zz is null or |z| = 0).
__device__ __forceinline__ double fd_eps(const double *eps_p, const double *zz) {
  const double eps_num = eps_p ? *eps_p : 0.;
  if (!zz) return eps_num;
  const double q = *zz;
  return q > 0. ? eps_num / sqrt(q) : eps_num;
}
template <class T>
__global__ void k_load_state(int nc, int nt, const double *__restrict__ Wn, const T *__restrict__ dir,
                             const double *__restrict__ eps_num, const double *__restrict__ zz, double *__restrict__ W) {
  pdl_wait();
  pdl_trigger();
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  const double eps = dir ? fd_eps(eps_num, zz) : 0.;
#pragma unroll
  for (int v = 0; v < 5; ++v) W[v * nt + c] = Wn[v * nc + c] + (dir ? eps * double(dir[v * nc + c]) : 0.);
}
template <class T, class D>
__global__ void k_load_dual(int nc, int nt, const double *__restrict__ Wn, const T *__restrict__ dir, Dual<D> *__restrict__ W) {
  pdl_wait();
  pdl_trigger();
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
#pragma unroll
  for (int v = 0; v < 5; ++v) W[v * nt + c] = Dual<D>(D(Wn[v * nc + c]), D(dir[v * nc + c]));
}

// y = (V P/dt) z - Jz, Jz from a finite difference (R1 - R0)/eps or a tangent run
template <class T, class D = double>
__global__ void k_matvec_finish(DevCase cs, int nc, const double *__restrict__ Wn, const double *__restrict__ vol,
                                const double *__restrict__ dt, const T *__restrict__ z, const double *__restrict__ R1,
                                const double *__restrict__ R0, const IterConsts *__restrict__ ic, const double *__restrict__ zz,
                                const Dual<D> *__restrict__ JV, T *__restrict__ y) {
  pdl_wait();
  pdl_trigger();
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  const double inv_eps = JV ? 0. : 1. / fd_eps(&ic->eps_num, zz);
  double P[25];
  cons2prim(cs, Wn[c], Wn[nc + c], Wn[2 * nc + c], Wn[3 * nc + c], Wn[4 * nc + c], P);
  const double s = vol[c] / dt[c];
  double zv[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) zv[k] = double(z[k * nc + c]);
#pragma unroll
  for (int i = 0; i < 5; ++i) {
    double a = 0.;
#pragma unroll
    for (int k = 0; k < 5; ++k) a += P[5 * i + k] * zv[k];
    const double jz = JV ? double(JV[i * nc + c].d) : (R1[i * nc + c] - R0[i * nc + c]) * inv_eps;
    y[i * nc + c] = T(ic->rs.s[i] * (s * a - jz));
  }
}

// ------------------------------------------------------------------ Krylov vector kernels
constexpr int kRedBlocks = 592;  // 4 x 148

__device__ void last_block_sum(int nparts, const double *part, double *__restrict__ out, unsigned *__restrict__ count);
template <class T>
__global__ void k_dots(int n, int nv, const T *__restrict__ V, size_t ld, const T *__restrict__ w, double *__restrict__ part,
                       double *__restrict__ out = nullptr, unsigned *__restrict__ count = nullptr) {
  pdl_wait();
  pdl_trigger();
  // part[v*gridDim.x + block] = sum over this block's slice of V_v . w; with
  // counters (one per column, blockDim == 256) the column's last block also
  // writes out[v]
  const int v = blockIdx.y;
  const T *a = V + (size_t)v * ld;
  double s = 0.;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) s += double(a[i]) * double(w[i]);
  __shared__ double sh[32];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += sh[k];
    part[v * gridDim.x + blockIdx.x] = t;
  }
  if (count) last_block_sum(gridDim.x, part + (size_t)v * gridDim.x, out + v, count + v);
  (void)nv;
}
__global__ void k_sum_parts(int nparts, const double *__restrict__ part, double *__restrict__ out) {
  pdl_wait();
  pdl_trigger();
  const int v = blockIdx.x;
  double s = 0.;
  for (int i = threadIdx.x; i < nparts; i += blockDim.x) s += part[v * nparts + i];
  __shared__ double sh[32];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += sh[k];
    out[v] = t;
  }
}
// w -= sum_v h[v] V_v
template <class T>
__global__ void k_sub_combo(int n, int nv, const T *__restrict__ V, size_t ld, const double *__restrict__ h, T *__restrict__ w) {
  pdl_wait();
  pdl_trigger();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double s = double(w[i]);
  for (int v = 0; v < nv; ++v) s -= h[v] * double(V[(size_t)v * ld + i]);
  w[i] = T(s);
}
// out = sum_v y[v] V_v
template <class T>
__global__ void k_combo(int n, int nv, const T *__restrict__ V, size_t ld, const double *__restrict__ y, T *__restrict__ out) {
  pdl_wait();
  pdl_trigger();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double s = 0.;
  for (int v = 0; v < nv; ++v) s += y[v] * double(V[(size_t)v * ld + i]);
  out[i] = T(s);
}
template <class T>
__global__ void k_scale_copy(int n, const double *__restrict__ a, double alpha, T *__restrict__ b) {
  pdl_wait();
  pdl_trigger();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = T(alpha * a[i]);
}
template <class T>
__global__ void k_scale(int n, double alpha, T *__restrict__ b) {
  pdl_wait();
  pdl_trigger();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = T(alpha * double(b[i]));
}
// W += alpha dW with a NaN/Inf check (update_variables, ns.cc:338-356)
template <class T>
__global__ void k_update(int n, double *__restrict__ Wn, const T *__restrict__ dW, double alpha, int *__restrict__ err) {
  pdl_wait();
  pdl_trigger();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double d = double(dW[i]);
  if (!isfinite(d)) atomicOr(err, 8);
  Wn[i] += alpha * d;
}
// scaled copy b = alpha a (same type)
__global__ void k_rowscale_copy(int nc, const double *__restrict__ a, RowScale rs, double alpha, double *__restrict__ b) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  for (int v = 0; v < 5; ++v) b[v * nc + c] = alpha * rs.s[v] * a[v * nc + c];
}
// largest relative change of the absolute pressure and temperature, as an ordered key
__global__ void k_max_rel_change(DevCase cs, int nc, const double *__restrict__ Wn, const double *__restrict__ dW,
                                 unsigned long long *__restrict__ key) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  double r = 0.;
  if (c < nc) {
    const double pa = Wn[c] + cs.Pref, Ta = Wn[4 * nc + c] + cs.Tref;
    const double rp = ::fabs(dW[c]) / ::fabs(pa), rT = ::fabs(dW[4 * nc + c]) / ::fabs(Ta);
    r = rp > rT ? rp : rT;
    if (!isfinite(r)) r = 1e300;
  }
  for (int o = 16; o > 0; o >>= 1) r = fmax(r, __shfl_xor_sync(0xffffffffu, r, o));
  if ((threadIdx.x & 31) == 0) atomicMax(key, okey(r));
}
// Explicit start-up step per cell: (V P / dt) dW = R (the time-term block of
// the implicit operator alone: forward Euler in the primitive variables with
// the local time step), W += dW, a non-finite dW flagged (err bit 8).  The
// 5x5 system is solved by Gaussian elimination with partial pivoting.
__global__ void k_explicit_update(DevCase cs, int nc, double *__restrict__ Wn, const double *__restrict__ R,
                                  const double *__restrict__ vol, const double *__restrict__ dt, int *__restrict__ err) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  double A[25], b[5];
  cons2prim(cs, Wn[c], Wn[nc + c], Wn[2 * nc + c], Wn[3 * nc + c], Wn[4 * nc + c], A);
  const double s = vol[c] / dt[c];
#pragma unroll
  for (int i = 0; i < 25; ++i) A[i] *= s;
#pragma unroll
  for (int i = 0; i < 5; ++i) b[i] = R[(size_t)i * nc + c];
  for (int k = 0; k < 5; ++k) {
    int piv = k;
    for (int i = k + 1; i < 5; ++i)
      if (::fabs(A[5 * i + k]) > ::fabs(A[5 * piv + k])) piv = i;
    if (piv != k) {
      for (int j = 0; j < 5; ++j) { const double t = A[5 * k + j]; A[5 * k + j] = A[5 * piv + j]; A[5 * piv + j] = t; }
      const double t = b[k]; b[k] = b[piv]; b[piv] = t;
    }
    for (int i = k + 1; i < 5; ++i) {
      const double f = A[5 * i + k] / A[5 * k + k];
      for (int j = k; j < 5; ++j) A[5 * i + j] -= f * A[5 * k + j];
      b[i] -= f * b[k];
    }
  }
  double d[5];
  for (int i = 4; i >= 0; --i) {
    double t = b[i];
    for (int j = i + 1; j < 5; ++j) t -= A[5 * i + j] * d[j];
    d[i] = t / A[5 * i + i];
  }
  bool bad = false;
#pragma unroll
  for (int i = 0; i < 5; ++i) bad = bad || !isfinite(d[i]);
  if (bad) {
    atomicOr(err, 8);
    return;
  }
#pragma unroll
  for (int i = 0; i < 5; ++i) Wn[(size_t)i * nc + c] += d[i];
}
// W += a_c dW per cell, a_c = min(1, 0.2 / max(|dp|/|p|, |dT|/|T|)) (absolute
// p, T), with the NaN/Inf check of k_update
__global__ void k_update_local(DevCase cs, int nc, double *__restrict__ Wn, const double *__restrict__ dW,
                               int *__restrict__ err) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  const double pa = Wn[c] + cs.Pref, Ta = Wn[4 * nc + c] + cs.Tref;
  const double rp = ::fabs(dW[c]) / ::fabs(pa), rT = ::fabs(dW[4 * nc + c]) / ::fabs(Ta);
  const double r = rp > rT ? rp : rT;
  if (!isfinite(r)) {
    atomicOr(err, 8);
    return;
  }
  const double a = r > 0.2 ? 0.2 / r : 1.;
  for (int v = 0; v < 5; ++v) Wn[(size_t)v * nc + c] += a * dW[(size_t)v * nc + c];
}
__global__ void k_aos_to_soa_nc(const double *__restrict__ in, double *__restrict__ out, int nc) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  for (int v = 0; v < 5; ++v) out[v * nc + c] = in[5 * c + v];
}
__global__ void k_soa_to_aos_nc(const double *__restrict__ in, double *__restrict__ out, int nc) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  for (int v = 0; v < 5; ++v) out[5 * c + v] = in[v * nc + c];
}
__global__ void k_gather_vol(int nc, const double *__restrict__ v, double *__restrict__ out) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < nc) out[c] = v[c];
}

// ------------------------------------------------------------------ solver
// Second pass of a dot product inside the kernel that wrote its block
// partials: the block of column v that finishes last adds part[0..nparts)
// exactly as k_sum_parts does (same thread strides, shuffles and warp order,
// so the sum is bit-identical) and re-arms the column's counter for the next
// launch.  Blocks of kFusedThreads threads.
constexpr int kFusedThreads = 256;
__device__ void last_block_sum(int nparts, const double *part, double *__restrict__ out, unsigned *__restrict__ count) {
  __shared__ unsigned ticket;
  __shared__ double shs[kFusedThreads / 32];
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) ticket = atomicAdd(count, 1u);
  __syncthreads();
  if (ticket != (unsigned)nparts - 1u) return;
  __threadfence();
  double s = 0.;
  for (int i = threadIdx.x; i < nparts; i += kFusedThreads) s += __ldcg(part + i);
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) shs[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.;
    for (int k = 0; k < kFusedThreads / 32; ++k) t += shs[k];
    *out = t;
    *count = 0u;
  }
}

// part[block] = sum over this block's slice of (z_i / wref_v)^2, v = i / nc
template <class T>
__global__ void k_wdot(int n, int nc, const T *__restrict__ z, const RowScale *__restrict__ winv, double *__restrict__ part,
                       double *__restrict__ out = nullptr, unsigned *__restrict__ count = nullptr) {
  pdl_wait();
  pdl_trigger();
  double s = 0.;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double q = double(z[i]) * winv->s[i / nc];
    s += q * q;
  }
  __shared__ double sh[32];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += sh[k];
    part[blockIdx.x] = t;
  }
  // with a counter (blockDim == kFusedThreads): the last block also forms the sum
  if (count) last_block_sum(gridDim.x, part, out, count);
}

template <class T>
__global__ void k_scale_rsqrt(int n, const double *__restrict__ ss, T *__restrict__ b) {
  pdl_wait();
  pdl_trigger();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const double q = *ss;
  if (i < n && q > 0.) b[i] = T(double(b[i]) / sqrt(q));
}


template <class T>
struct Krylov {
  fcfd_ctx *x = nullptr;
  int n = 0, nc = 0, m = 0, nparts = 1;
  DBuf<T> V, w, tmpT;
  DBuf<double> part, hd;  // hd: [0,m+1) first CGS pass, [m+1,2m+2) second, [2m+2] |w|^2, [2m+3] |z|^2
  DBuf<unsigned> count;   // per-column arrival counters of the single-launch dot products (re-armed by each launch)
  double *hp = nullptr;   // pinned host mirror of hd
  // one CUDA graph per basis index j of the Arnoldi step (preconditioner,
  // J.v, both Gram-Schmidt passes, normalisation, copy of hd to hp),
  // captured at its first use and replayed for every later cycle and Newton
  // step of the solve
  std::vector<cudaGraphExec_t> graphs;
  Krylov() = default;
  Krylov(const Krylov &) = delete;
  Krylov &operator=(const Krylov &) = delete;
  ~Krylov() {
    for (cudaGraphExec_t g : graphs)
      if (g) cudaGraphExecDestroy(g);
    if (hp) cudaFreeHost(hp);
  }
  void alloc(fcfd_ctx *ctx, int krylov_dim) {
    x = ctx; nc = ctx->dm.nc; n = 5 * nc; m = krylov_dim;
    nparts = std::min(kRedBlocks, std::max(1, (n + 1023) / 1024));
    V.alloc((size_t)(m + 1) * n); w.alloc(n); tmpT.alloc(n);
    part.alloc((size_t)nparts * (m + 1)); hd.alloc(2 * (size_t)m + 4); count.alloc(m + 1);
    CK(cudaMemsetAsync(count.p, 0, sizeof(unsigned) * (m + 1), x->stream));
    CK(cudaMallocHost((void **)&hp, sizeof(double) * (2 * (size_t)m + 4)));
    graphs.assign(m, nullptr);
  }
  double *h1() { return hd.p; }
  double *h2() { return hd.p + m + 1; }
  double *ww() { return hd.p + 2 * m + 2; }
  double *zz() { return hd.p + 2 * m + 3; }
  // out[v] = Vb_v . u for v < nv, left on the device (deterministic two-pass reduction)
  void dots_dev(int nv, const T *Vb, const T *u, double *out) {
    cudaStream_t s = x->stream;
    dim3 g(nparts, nv);
    k_dots<T><<<g, 256, 0, s>>>(n, nv, Vb, (size_t)n, u, part.p);
    k_sum_parts<<<nv, 256, 0, s>>>(nparts, part.p, out);
  }
  // out[v] = Vb_v . u for v < nv in one launch (the column's last block adds the partials)
  void dots_fused(int nv, const T *Vb, const T *u, double *out) {
    launch_k(x->pdl, k_dots<T>, dim3(nparts, nv), kFusedThreads, 0, x->stream, n, nv, Vb, (size_t)n, u, part.p, out,
             count.p);
  }
  // bring hd back to the host (the one synchronisation of a GMRES iteration)
  void fetch_async() {
    CK(cudaMemcpyAsync(hp, hd.p, sizeof(double) * (2 * (size_t)m + 4), cudaMemcpyDeviceToHost, x->stream));
  }
  void fetch() {
    fetch_async();
    CK(cudaStreamSynchronize(x->stream));
  }
  double norm(const T *u) {
    dots_dev(1, u, u, ww());
    fetch();
    return std::sqrt(hp[2 * m + 2]);
  }
  // |S^-1 u|^2 on the device (S = per-variable reference magnitudes)
  void wnorm2_dev(const T *u, const RowScale *winv, double *out) {
    cudaStream_t s = x->stream;
    launch_k(x->pdl, k_wdot<T>, nparts, kFusedThreads, 0, s, n, nc, u, winv, part.p, out, count.p);
  }
  double norm64(const double *u) {
    cudaStream_t s = x->stream;
    k_dots<double><<<dim3(nparts, 1), 256, 0, s>>>(n, 1, u, (size_t)n, u, part.p);
    k_sum_parts<<<1, 256, 0, s>>>(nparts, part.p, ww());
    fetch();
    return std::sqrt(hp[2 * m + 2]);
  }
};

struct NewtonState {
  DBuf<double> Wn, R0, R1, dt, vol, JL, JR, Minv, Pr, Py0, Py1, Xs, rowmag;
  DBuf<double> OB, MinvP;  // couplings packed per colour for the Gauss-Seidel sweeps
  // FP32 copies for the mixed-precision preconditioner (fp32_krylov)
  DBuf<float> OB32, MinvP32, Pr32, Py32;
  bool prec32 = false;
  double wscale = 1.;  // |S^-1 W| (finite-difference step scale)
  RowScale winv;       // 1 / per-variable reference magnitudes
  int sweeps = 0, cycles = 1;
  IterConsts hic;      // host copy of the iteration scalars
  DBuf<IterConsts> ic; // their device copy
  // persistent Gauss-Seidel launch (k_gs_persist): on when the options ask
  // for it and the colouring fits its limits
  bool gs_persist = false, gs_stage = false;
  int gs_blocks = 0, gs_dmax = 0;  // gs_dmax: neighbour slots the kernel is compiled for (4 or kGsMaxDeg)
  size_t gs_smem = 0;
  GsPersistArgs gs_args{};
  DBuf<int> gs_sched;
  DBuf<unsigned> gs_bar;  // [0] barrier arrivals, [1] timeout flag
  // block ILU(0) in the multicolour order: the modified diagonal inverses by
  // cell and every cell's colour; the solve is one symmetric colour sweep
  // from y = 0 with those inverses
  bool ilu = false;
  DBuf<double> MinvT;
  DBuf<int> colour;
};

// Colour of every Gauss-Seidel update of one preconditioner application with
// `sweeps` symmetric sweeps: colours forward, then backward, skipping a
// colour that would be updated twice in a row (no change) and empty colours.
static std::vector<int> gs_schedule(const std::vector<int> &ci, int sweeps) {
  const int ncol = (int)ci.size() - 1;
  std::vector<int> out;
  int last = -1;
  for (int k = 0; k < sweeps; ++k)
    for (int pass = 0; pass < 2; ++pass)
      for (int q = 0; q < ncol; ++q) {
        const int col = pass == 0 ? q : ncol - 1 - q;
        if (ci[col + 1] - ci[col] <= 0 || col == last) continue;
        last = col;
        out.push_back(col);
      }
  return out;
}

// Grid size, shared memory and staging of k_gs_persist for couplings of type
// P: one block per SM with the couplings staged when they fit in shared
// memory, else as many co-resident blocks as the occupancy allows (at least
// 32 cells of the largest colour per block).
template <class P>
static void plan_gs_persist(fcfd_ctx *x, NewtonState &ns) {
  const std::vector<int> &ci = x->color_index;
  const int ncol = (int)ci.size() - 1, deg = x->gs_deg;
  if (ncol < 1 || ncol > kGsMaxCol || deg < 1 || deg > kGsMaxDeg) return;
  const std::vector<int> sched = gs_schedule(ci, ns.sweeps);
  if (sched.empty()) return;
  int nsm = 0, coop = 0, optin = 0;
  CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, x->device));
  CK(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, x->device));
  CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, x->device));
  if (!coop || nsm < 1) return;
  int maxcnt = 0;
  for (int col = 0; col < ncol; ++col) maxcnt = std::max(maxcnt, ci[col + 1] - ci[col]);
  const int need = std::max(1, (maxcnt + 31) / 32);
  const size_t ts_bytes = sizeof(P) * 5 * 32 * kGsZ;
  auto chunks = [&](int nb, int *soff) {
    soff[0] = 0;
    for (int col = 0; col < ncol; ++col) soff[col + 1] = soff[col] + (ci[col + 1] - ci[col] + nb - 1) / nb;
    return soff[ncol];
  };
  GsPersistArgs &a = ns.gs_args;
  a.nc = x->dm.nc; a.deg = deg; a.ncol = ncol; a.nphase = (int)sched.size();
  a.cells = x->color_cells.p; a.nbr = x->gs_nbr.p;
  for (int col = 0; col <= ncol; ++col) a.cidx[col] = ci[col];
  const int threads = 32 * 5 * kGsZ;
  int nb = std::min(nsm, need);
  const int stot = chunks(nb, a.soff);
  const size_t stage_bytes = ts_bytes + (size_t)stot * ((size_t)deg * 25 + 30) * sizeof(P) + (size_t)stot * (1 + deg) * sizeof(int);
  int occ = 0;
  ns.gs_dmax = deg <= 4 ? 4 : kGsMaxDeg;
  auto kern = [&](bool stage) -> const void * {
    if (ns.gs_dmax == 4) return stage ? (const void *)k_gs_persist<P, true, 4> : (const void *)k_gs_persist<P, false, 4>;
    return stage ? (const void *)k_gs_persist<P, true, kGsMaxDeg> : (const void *)k_gs_persist<P, false, kGsMaxDeg>;
  };
  if (stage_bytes <= (size_t)optin) {
    CK(cudaFuncSetAttribute(kern(true), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)stage_bytes));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern(true), threads, stage_bytes));
    if (occ >= 1) {
      ns.gs_stage = true;
      ns.gs_smem = stage_bytes;
    }
  }
  if (!ns.gs_stage) {
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern(false), threads, ts_bytes));
    if (occ < 1) return;
    nb = std::min(nsm * occ, need);
    chunks(nb, a.soff);
    ns.gs_smem = ts_bytes;
  }
  ns.gs_blocks = nb;
  ns.gs_sched.upload(sched);
  ns.gs_bar.alloc(2);
  CK(cudaMemsetAsync(ns.gs_bar.p, 0, 2 * sizeof(unsigned), x->stream));
  a.sched = ns.gs_sched.p;
  a.bar = ns.gs_bar.p;
  ns.gs_persist = true;
}

template <class P>
static void launch_gs_persist(fcfd_ctx *x, NewtonState &ns, const P *OB, const P *MinvP, const P *r, P *y) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(ns.gs_blocks);
  cfg.blockDim = dim3(32, 5, kGsZ);
  cfg.dynamicSmemBytes = ns.gs_smem;
  cfg.stream = x->stream;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeCooperative;
  at[0].val.cooperative = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  if (ns.gs_dmax == 4) {
    if (ns.gs_stage) CK(cudaLaunchKernelEx(&cfg, k_gs_persist<P, true, 4>, ns.gs_args, OB, MinvP, r, y));
    else CK(cudaLaunchKernelEx(&cfg, k_gs_persist<P, false, 4>, ns.gs_args, OB, MinvP, r, y));
  } else {
    if (ns.gs_stage) CK(cudaLaunchKernelEx(&cfg, k_gs_persist<P, true, kGsMaxDeg>, ns.gs_args, OB, MinvP, r, y));
    else CK(cudaLaunchKernelEx(&cfg, k_gs_persist<P, false, kGsMaxDeg>, ns.gs_args, OB, MinvP, r, y));
  }
}

// FCFD_ERR_TIMEOUT if a grid barrier of the persistent Gauss-Seidel kernel ran
// out of polls since the last check (the flag is cleared)
static void check_gs_timeout(fcfd_ctx *x, NewtonState &ns) {
  if (!ns.gs_persist) return;
  unsigned h = 0;
  CK(cudaMemcpyAsync(&h, ns.gs_bar.p + 1, sizeof(unsigned), cudaMemcpyDeviceToHost, x->stream));
  CK(cudaStreamSynchronize(x->stream));
  if (h) {
    CK(cudaMemsetAsync(ns.gs_bar.p + 1, 0, sizeof(unsigned), x->stream));
    throw Error(FCFD_ERR_TIMEOUT, "a grid barrier of the persistent Gauss-Seidel kernel timed out");
  }
}
template <class T>
__global__ void k_axpy_to(int n, const double *__restrict__ b, const T *__restrict__ w, T *__restrict__ out) {
  pdl_wait();
  pdl_trigger();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = T(b[i] - double(w[i]));
}
template <class T, class A = double>
__global__ void k_cast(int n, const A *__restrict__ a, T *__restrict__ b) {
  pdl_wait();
  pdl_trigger();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = T(a[i]);
}

// residual of the [5][nc] state (+ eps*dir) into R (SoA [5][nc])
template <class T>
static void eval_residual(fcfd_ctx *x, const double *Wn, double *R, const T *dir, const double *eps,
                          const double *zz = nullptr) {
  const DevMesh &m = x->dm;
  launch_k(x->pdl, k_load_state<T>, (m.nc + 255) / 256, 256, 0, x->stream, m.nc, m.nt, Wn, dir, eps, zz, x->p64.W.p);
  launch_chain<double>(x, x->p64, R, false, nullptr, nullptr);
}

// Tangent-chain buffers of the J.v mode, allocated before any capture.
static void prepare_matvec(fcfd_ctx *x, int mode) {
  const DevMesh &m = x->dm;
  if (mode == 0) return;
  if (x->newton_f32) {
    if (!x->pjv32.ready) x->pjv32.alloc(m.nc, m.nf, m.nb);
  } else {
    if (!x->pjv.ready) x->pjv.alloc(m.nc, m.nf, m.nb);
  }
}

// y = (V P/dt - dR/dW) z; zz: device |z|^2 (finite-difference mode only).
// Finite differences are taken in variables scaled by their reference
// magnitudes: eps = sqrt(eps_mach) (1 + |S^-1 W|) / |S^-1 z|, the numerator
// in ns.ic.
template <class T>
static void matvec(fcfd_ctx *x, NewtonState &ns, int mode, const T *z, T *y, const double *zz) {
  const DevMesh &m = x->dm;
  cudaStream_t s = x->stream;
  const int tb = 256, gb = (m.nc + tb - 1) / tb;
  prepare_matvec(x, mode);
  if (mode == 0) {
    eval_residual<T>(x, ns.Wn.p, ns.R1.p, z, &ns.ic.p->eps_num, zz);
    launch_k(x->pdl, k_matvec_finish<T, double>, gb, tb, 0, s, x->cs, m.nc, ns.Wn.p, ns.vol.p, ns.dt.p, z, ns.R1.p,
             ns.R0.p, ns.ic.p, zz, (const Dual<double> *)nullptr, y);
  } else {
    if (x->newton_f32) {
      launch_k(x->pdl, k_load_dual<T, float>, gb, tb, 0, s, m.nc, m.nt, ns.Wn.p, z, x->pjv32.W.p);
      launch_chain<Dual<float>>(x, x->pjv32, x->pjv32.R.p, false, nullptr, nullptr, x->newton_frozen);
      launch_k(x->pdl, k_matvec_finish<T, float>, gb, tb, 0, s, x->cs, m.nc, ns.Wn.p, ns.vol.p, ns.dt.p, z,
               (const double *)nullptr, (const double *)nullptr, ns.ic.p, (const double *)nullptr,
               (const Dual<float> *)x->pjv32.R.p, y);
    } else {
      launch_k(x->pdl, k_load_dual<T, double>, gb, tb, 0, s, m.nc, m.nt, ns.Wn.p, z, x->pjv.W.p);
      launch_chain<Dual<double>>(x, x->pjv, x->pjv.R.p, false, nullptr, nullptr, x->newton_frozen);
      launch_k(x->pdl, k_matvec_finish<T, double>, gb, tb, 0, s, x->cs, m.nc, ns.Wn.p, ns.vol.p, ns.dt.p, z,
               (const double *)nullptr, (const double *)nullptr, ns.ic.p, (const double *)nullptr,
               (const Dual<double> *)x->pjv.R.p, y);
    }
  }
  CK(cudaGetLastError());
}

static double dnorm(fcfd_ctx *x, DBuf<double> &part, DBuf<double> &h, const double *u, int n) {
  cudaStream_t s = x->stream;
  dim3 g(kRedBlocks, 1);
  k_dots<double><<<g, 256, 0, s>>>(n, 1, u, (size_t)n, u, part.p);
  k_sum_parts<<<1, 256, 0, s>>>(kRedBlocks, part.p, h.p);
  double r;
  CK(cudaMemcpyAsync(&r, h.p, sizeof(double), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  return std::sqrt(r);
}

// Preconditioner: z = M^-1 D^-1 v with M^-1 = `sweeps` symmetric multicolour
// block Gauss-Seidel sweeps on the first-order operator (0: block diagonal alone).
template <class T>
static void apply_prec(fcfd_ctx *x, NewtonState &ns, const T *v, T *z, int sweeps) {
  const int nc = x->dm.nc, tb = 256, gc = (nc + tb - 1) / tb;
  cudaStream_t s = x->stream;
  const RowScale *rs = &ns.ic.p->rs;
  if (sweeps <= 0) {
    launch_k(x->pdl, k_precond<T>, gc, tb, 0, s, nc, (const double *)ns.Minv.p, v, z, rs);
    return;
  }
  // r = D^-1 v, y0 = Binv r; then symmetric multicolour block Gauss-Seidel:
  // colours forward, then backward.  Updating the same colour twice in a row
  // changes nothing (its cells do not couple to each other), so the repeat at
  // each turn is skipped.  FP64 or, with the FP32 preconditioner, FP32
  // couplings, vectors and arithmetic.
  auto sweep = [&](auto *OB, auto *MinvP, auto *r, auto *a) {
    if (ns.gs_persist) {
      launch_gs_persist(x, ns, OB, MinvP, r, a);
      return;
    }
    const std::vector<int> &ci = x->color_index;
    const int ncol = (int)ci.size() - 1, deg = x->gs_deg;
    int last = -1;
    for (int k = 0; k < sweeps; ++k) {
      for (int pass = 0; pass < 2; ++pass)
        for (int q = 0; q < ncol; ++q) {
          const int col = pass == 0 ? q : ncol - 1 - q;
          const int cnt = ci[col + 1] - ci[col];
          if (cnt <= 0 || col == last) continue;
          last = col;
          const size_t base = (size_t)ci[col];
          launch_k(x->pdl, k_gs_rows<std::remove_const_t<std::remove_pointer_t<decltype(a)>>>, dim3((cnt + 31) / 32),
                   dim3(32, 5), 0, s, nc, deg, cnt, (const int *)(x->color_cells.p + base),
                   (const int *)(x->gs_nbr.p + base * deg), (const decltype(+*a) *)(OB + base * deg * 25),
                   (const decltype(+*a) *)(MinvP + base * 25), (const decltype(+*a) *)r, a);
        }
    }
  };
  // the sweeps run in place on z itself when it has the preconditioner's type
  auto run = [&](auto *OB, auto *MinvP, auto *r, auto *y) {
    using P = std::remove_pointer_t<decltype(y)>;
    unsigned *bar = ns.gs_persist ? ns.gs_bar.p : nullptr;
    if constexpr (std::is_same_v<P, T>) {
      launch_k(x->pdl, k_precond_split<T, P>, gc, tb, 0, s, nc, (const double *)ns.Minv.p, v, rs, r, z, bar);
      // ILU(0): the forward colour sweep starts from y = 0
      if (ns.ilu) CK(cudaMemsetAsync(z, 0, sizeof(P) * 5 * (size_t)nc, s));
      sweep(OB, MinvP, r, z);
    } else {
      launch_k(x->pdl, k_precond_split<T, P>, gc, tb, 0, s, nc, (const double *)ns.Minv.p, v, rs, r, y, bar);
      if (ns.ilu) CK(cudaMemsetAsync(y, 0, sizeof(P) * 5 * (size_t)nc, s));
      sweep(OB, MinvP, r, y);
      launch_k(x->pdl, k_cast<T, P>, (5 * nc + tb - 1) / tb, tb, 0, s, 5 * nc, (const P *)y, z);
    }
  };
  if (ns.prec32)
    run(ns.OB32.p, ns.MinvP32.p, ns.Pr32.p, ns.Py32.p);
  else
    run(ns.OB.p, ns.MinvP.p, ns.Pr.p, ns.Py0.p);
}

// dW = NaN: the update of a step whose right-hand side is not finite, so
// that the NaN check of the update reports the divergence (the reference's
// linear solve propagates the NaN into its update, ns.cc:349-355)
__global__ void k_fill_nan(int n, double *__restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = __longlong_as_double(0x7ff8000000000000ll);
}

// Right-preconditioned GMRES(m) with up to `cycles` restarts.
template <class T>
static void gmres(fcfd_ctx *x, NewtonState &ns, Krylov<T> &K, int mode, double rtol, double *dW, int &iters, double &relres,
                  const RowScale &rs, double abstol = 0.) {
  const int n = K.n, m = K.m, nc = K.nc;
  cudaStream_t s = x->stream;
  const int tb = 256, gn = (n + tb - 1) / tb, gc = (nc + tb - 1) / tb;
  iters = 0;
  relres = 1.;
  prepare_matvec(x, mode);
  // scaled right-hand side b = D R0; x0 = 0
  k_rowscale_copy<<<gc, tb, 0, s>>>(nc, ns.R0.p, rs, 1., dW);
  const double bnorm = K.norm64(dW);
  CK(cudaMemsetAsync(ns.Xs.p, 0, sizeof(double) * n, s));
  if (!std::isfinite(bnorm)) {
    k_fill_nan<<<gn, tb, 0, s>>>(n, dW);
    relres = bnorm;
    return;
  }
  if (!(bnorm > 0.)) { CK(cudaMemsetAsync(dW, 0, sizeof(double) * n, s)); relres = 0.; return; }
  std::vector<double> H((size_t)(m + 1) * m, 0.), cs(m), sn(m), g(m + 1, 0.);
  for (int cyc = 0; cyc < ns.cycles; ++cyc) {
    double beta;
    if (cyc == 0) {
      beta = bnorm;
      k_scale_copy<T><<<gn, tb, 0, s>>>(n, dW, 1. / beta, K.V.p);
    } else {
      // r = b - (D A M^-1 D^-1 ...) applied to the current solution: recompute through one matvec of
      // z = M^-1 D^-1 (sum) already folded into Xs (physical units): r = D (R0 - A Xs)
      k_cast<T><<<gn, tb, 0, s>>>(n, ns.Xs.p, K.tmpT.p);
      if (mode == 0) K.wnorm2_dev(K.tmpT.p, &ns.ic.p->winv, K.zz());
      matvec<T>(x, ns, mode, K.tmpT.p, K.w.p, K.zz());
      k_rowscale_copy<<<gc, tb, 0, s>>>(nc, ns.R0.p, rs, 1., dW);
      k_axpy_to<T><<<gn, tb, 0, s>>>(n, dW, K.w.p, K.V.p);  // V0 = b - A x (unnormalised)
      beta = K.norm(K.V.p);
      if (!(beta > 0.)) break;
      k_scale<T><<<gn, tb, 0, s>>>(n, 1. / beta, K.V.p);
    }
    std::fill(g.begin(), g.end(), 0.);
    g[0] = beta;
    int k = 0;
    bool done = false;
    for (int j = 0; j < m; ++j) {
      if (!K.graphs[j]) {
        T *vj = K.V.p + (size_t)j * n;
        T *w = K.V.p + (size_t)(j + 1) * n;
        cudaGraph_t gr = nullptr;
        CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        apply_prec<T>(x, ns, vj, K.tmpT.p, ns.sweeps);
        if (mode == 0) K.wnorm2_dev(K.tmpT.p, &ns.ic.p->winv, K.zz());
        matvec<T>(x, ns, mode, K.tmpT.p, w, K.zz());
        // classical Gram-Schmidt twice, coefficients kept on the device
        K.dots_fused(j + 1, K.V.p, w, K.h1());
        launch_k(x->pdl, k_sub_combo<T>, gn, tb, 0, s, n, j + 1, (const T *)K.V.p, (size_t)n, (const double *)K.h1(), w);
        K.dots_fused(j + 1, K.V.p, w, K.h2());
        launch_k(x->pdl, k_sub_combo<T>, gn, tb, 0, s, n, j + 1, (const T *)K.V.p, (size_t)n, (const double *)K.h2(), w);
        K.dots_fused(1, w, w, K.ww());
        launch_k(x->pdl, k_scale_rsqrt<T>, gn, tb, 0, s, n, (const double *)K.ww(), w);
        K.fetch_async();
        CK(cudaStreamEndCapture(s, &gr));
        CK(cudaGraphInstantiate(&K.graphs[j], gr, 0));
        CK(cudaGraphDestroy(gr));
      }
      CK(cudaGraphLaunch(K.graphs[j], s));
      CK(cudaStreamSynchronize(s));
      const double hn = std::sqrt(K.hp[2 * m + 2]);
      for (int i = 0; i <= j; ++i) H[(size_t)i * m + j] = K.hp[i] + K.hp[m + 1 + i];
      H[(size_t)(j + 1) * m + j] = hn;
      for (int i = 0; i < j; ++i) {
        const double a = H[(size_t)i * m + j], b = H[(size_t)(i + 1) * m + j];
        H[(size_t)i * m + j] = cs[i] * a + sn[i] * b;
        H[(size_t)(i + 1) * m + j] = -sn[i] * a + cs[i] * b;
      }
      const double a = H[(size_t)j * m + j], b = H[(size_t)(j + 1) * m + j];
      const double r = std::hypot(a, b);
      cs[j] = (r > 0.) ? a / r : 1.;
      sn[j] = (r > 0.) ? b / r : 0.;
      H[(size_t)j * m + j] = r;
      H[(size_t)(j + 1) * m + j] = 0.;
      g[j + 1] = -sn[j] * g[j];
      g[j] = cs[j] * g[j];
      k = j + 1;
      ++iters;
      relres = std::fabs(g[j + 1]) / bnorm;
      if (relres <= rtol || std::fabs(g[j + 1]) <= abstol || !(hn > 0.)) { done = true; break; }
    }
    std::vector<double> y(k, 0.);
    for (int i = k - 1; i >= 0; --i) {
      double t = g[i];
      for (int l = i + 1; l < k; ++l) t -= H[(size_t)i * m + l] * y[l];
      y[i] = t / H[(size_t)i * m + i];
    }
    std::copy(y.begin(), y.end(), K.hp);
    CK(cudaMemcpyAsync(K.hd.p, K.hp, sizeof(double) * k, cudaMemcpyHostToDevice, s));
    k_combo<T><<<gn, tb, 0, s>>>(n, k, K.V.p, (size_t)n, K.hd.p, K.w.p);
    apply_prec<T>(x, ns, K.w.p, K.tmpT.p, ns.sweeps);
    k_update<T><<<gn, tb, 0, s>>>(n, ns.Xs.p, K.tmpT.p, 1., x->err.p);
    if (done) break;
  }
  CK(cudaMemcpyAsync(dW, ns.Xs.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
  CK(cudaGetLastError());
}

// Buffers of the implicit solve; volumes uploaded.
static void alloc_state(fcfd_ctx *x, NewtonState &ns, int sweeps, int cycles, bool prec32, int gs_launch = 0,
                        bool ilu = false) {
  const DevMesh &m = x->dm;
  const int nc = m.nc, n = 5 * nc;
  cudaStream_t s = x->stream;
  ns.Wn.alloc(n); ns.R0.alloc(n); ns.R1.alloc(n); ns.dt.alloc(nc); ns.vol.alloc(nc);
  ns.JL.alloc(25 * (size_t)m.nf); ns.JR.alloc(25 * (size_t)m.nf); ns.Minv.alloc(25 * (size_t)nc);
  ns.Pr.alloc(n); ns.Py0.alloc(n); ns.Py1.alloc(n); ns.Xs.alloc(n); ns.rowmag.alloc(n);
  ns.ic.alloc(1);
  ns.sweeps = sweeps; ns.cycles = cycles > 0 ? cycles : 1;
  ns.prec32 = prec32;
  ns.ilu = ilu && x->gs_deg > 0;
  if (ns.ilu) {
    // ILU(0): one forward and one backward colour sweep (the packed couplings
    // of the Gauss-Seidel path, the modified diagonal inverses)
    ns.sweeps = 1;
    ns.MinvT.alloc(25 * (size_t)nc);
    std::vector<int> colour(nc, 0);
    const std::vector<int> &ci = x->color_index;
    const std::vector<int32_t> &cc = x->mesh->color_cells;
    for (size_t col = 0; col + 1 < ci.size(); ++col)
      for (int k = ci[col]; k < ci[col + 1]; ++k) colour[cc[k]] = (int)col;
    ns.colour.upload(colour);
  }
  if (ns.sweeps > 0) {
    if (ns.prec32) {
      ns.OB32.alloc((size_t)nc * x->gs_deg * 25 + 1); ns.MinvP32.alloc(25 * (size_t)nc);
      ns.Pr32.alloc(5 * (size_t)nc); ns.Py32.alloc(5 * (size_t)nc);
    } else {
      ns.OB.alloc((size_t)nc * x->gs_deg * 25 + 1); ns.MinvP.alloc(25 * (size_t)nc);
    }
  }
  if (ns.sweeps > 0 && gs_launch == 1) {
    if (ns.prec32) plan_gs_persist<float>(x, ns);
    else plan_gs_persist<double>(x, ns);
  }
  CK(cudaMemsetAsync(ns.JR.p, 0, sizeof(double) * 25 * (size_t)m.nf, s));
  std::vector<double> vol(x->mesh->c_volume.begin(), x->mesh->c_volume.begin() + nc);
  CK(cudaMemcpyAsync(ns.vol.p, vol.data(), sizeof(double) * nc, cudaMemcpyHostToDevice, s));
  CK(cudaStreamSynchronize(s));
}

// First-order face Jacobians JL, JR [25][nf] at the state of the last residual
// chain run on x->p64 (states, gradients, limiters and stale densities).
// mutf: face eddy viscosities of a turbulent case (added to the viscosity of
// the viscous flux), or null.
static void launch_face_jac(fcfd_ctx *x, double *JL, double *JR, const double *mutf = nullptr) {
  const DevMesh &m = x->dm;
  cudaStream_t s = x->stream;
  if (x->viscous)
    FCFD_BY_FLUX(x->cs.flux, k_face_jac<true, FX><<<(m.nf + 127) / 128, 128, 0, s>>>(x->cs, m, x->p64.W.p, x->p64.G.p, x->p64.Lm.p, x->p64.stale.p, JL, JR, mutf));
  else
    FCFD_BY_FLUX(x->cs.flux, k_face_jac<false, FX><<<(m.nf + 127) / 128, 128, 0, s>>>(x->cs, m, x->p64.W.p, x->p64.G.p, x->p64.Lm.p, x->p64.stale.p, JL, JR, mutf));
}

// Inverse block-Jacobi blocks (V P/dt - J_cc)^-1 [25][nc] of the flow
// equations at the state of the last residual chain run on x->p64 (Wn its
// [5][nc] copy), with the face eddy viscosities mutf of a turbulent case
// (null: laminar).  JL, JR: [25][nf] scratch.  Used by the coupled k-omega
// Newton solve (rans.cu).
void ns_block_inverse(fcfd_ctx *x, const double *Wn, const double *vol, const double *dt, const double *mutf,
                      double *JL, double *JR, double *Minv, double *rowmag) {
  const DevMesh &m = x->dm;
  cudaStream_t s = x->stream;
  CK(cudaMemsetAsync(JR, 0, sizeof(double) * 25 * (size_t)m.nf, s));
  launch_face_jac(x, JL, JR, mutf);
  RowScale wref;
  for (int v = 0; v < 5; ++v) wref.s[v] = 1.;
  k_block_jacobi<<<(m.nc + 255) / 256, 256, 0, s>>>(x->cs, m, Wn, vol, dt, JL, JR, Minv, x->err.p, wref, rowmag);
  CK(cudaGetLastError());
}

// One linearised backward-Euler solve at the state the last residual loaded
// (ns.Wn, residual in ns.R0, local time step in ns.dt): the preconditioner
// from the first-order face Jacobians, then GMRES for (V P/dt - J) dW = R0 into
// ns.R1.  Shared by the Newton solve and the time-marching driver.
struct LinearSolve {
  int iters = 0;
  double relres = 0.;
};
static LinearSolve implicit_solve(fcfd_ctx *x, NewtonState &ns, Krylov<double> &K64, Krylov<float> &K32, bool f32, int jmode,
                                  double krtol, double abstol, DBuf<double> &part, DBuf<double> &hh) {
  const DevMesh &m = x->dm;
  const int nc = m.nc;
  cudaStream_t s = x->stream;
  const int tb = 256, gc = (nc + tb - 1) / tb;
  // reference state magnitudes: RMS of |p+Pref|, |V|, |T+Tref|
  RowScale wref;
  double wn[5];
  {
    double rp = dnorm(x, part, hh, ns.Wn.p, nc), ru = dnorm(x, part, hh, ns.Wn.p + nc, nc);
    double rv = dnorm(x, part, hh, ns.Wn.p + 2 * (size_t)nc, nc), rw = dnorm(x, part, hh, ns.Wn.p + 3 * (size_t)nc, nc);
    double rT = dnorm(x, part, hh, ns.Wn.p + 4 * (size_t)nc, nc);
    wn[0] = rp; wn[1] = ru; wn[2] = rv; wn[3] = rw; wn[4] = rT;
    const double sq = std::sqrt((double)nc);
    double U = std::sqrt(ru * ru + rv * rv + rw * rw) / sq;
    wref.s[0] = rp / sq + std::fabs(x->cs.Pref);
    wref.s[4] = rT / sq + std::fabs(x->cs.Tref);
    if (!(U > 0.)) U = std::sqrt(x->cs.gamma * x->cs.R * wref.s[4]);
    wref.s[1] = wref.s[2] = wref.s[3] = U;
  }
  // block-Jacobi preconditioner from the first-order face Jacobians
  launch_face_jac(x, ns.JL.p, ns.JR.p);
  k_block_jacobi<<<gc, tb, 0, s>>>(x->cs, m, ns.Wn.p, ns.vol.p, ns.dt.p, ns.JL.p, ns.JR.p, ns.Minv.p, x->err.p, wref, ns.rowmag.p);
  if (ns.sweeps > 0) {
    const std::vector<int> &ci = x->color_index;
    const int deg = x->gs_deg;
    if (ns.ilu) {
      for (size_t col = 0; col + 1 < ci.size(); ++col) {
        const int cnt = ci[col + 1] - ci[col];
        if (cnt <= 0) continue;
        const size_t base = (size_t)ci[col];
        k_ilu_diag<<<(cnt + 127) / 128, 128, 0, s>>>(x->cs, m, ns.Wn.p, ns.vol.p, ns.dt.p, ns.JL.p, ns.JR.p, deg, cnt,
                                                     (int)col, x->color_cells.p + base, x->gs_nbr.p + base * deg,
                                                     x->gs_src.p + base * deg, ns.colour.p, ns.MinvT.p, x->err.p);
      }
    }
    const double *Mpack = ns.ilu ? ns.MinvT.p : ns.Minv.p;
    for (size_t col = 0; col + 1 < ci.size(); ++col) {
      const int cnt = ci[col + 1] - ci[col];
      if (cnt <= 0) continue;
      const size_t base = (size_t)ci[col];
      if (ns.prec32)
        k_pack_gs<float><<<(cnt + 127) / 128, 128, 0, s>>>(nc, m.nf, deg, cnt, x->color_cells.p + base,
                                                           x->gs_nbr.p + base * deg, x->gs_src.p + base * deg, ns.JL.p,
                                                           ns.JR.p, Mpack, ns.OB32.p + base * deg * 25,
                                                           ns.MinvP32.p + base * 25);
      else
        k_pack_gs<double><<<(cnt + 127) / 128, 128, 0, s>>>(nc, m.nf, deg, cnt, x->color_cells.p + base,
                                                            x->gs_nbr.p + base * deg, x->gs_src.p + base * deg, ns.JL.p,
                                                            ns.JR.p, Mpack, ns.OB.p + base * deg * 25,
                                                            ns.MinvP.p + base * 25);
    }
  }
  CK(cudaGetLastError());
  // GMRES norm weights: 1 / RMS row magnitude, so every equation is measured
  // in units of a relative state change (consistent across equations)
  RowScale rs;
  for (int v = 0; v < 5; ++v) {
    const double r = dnorm(x, part, hh, ns.rowmag.p + (size_t)v * nc, nc) / std::sqrt((double)nc);
    rs.s[v] = (r > 0.) ? 1. / r : 1.;
  }
  for (int v = 0; v < 5; ++v) ns.winv.s[v] = 1. / wref.s[v];
  {
    // |S^-1 W| from the per-variable norms
    double q = 0.;
    for (int v = 0; v < 5; ++v) q += wn[v] * wn[v] * ns.winv.s[v] * ns.winv.s[v];
    ns.wscale = std::sqrt(q);
  }
  ns.hic.rs = rs;
  ns.hic.winv = ns.winv;
  for (int v = 0; v < 5; ++v) ns.hic.one.s[v] = 1.;
  ns.hic.eps_num = 1.4901161193847656e-08 * (1. + ns.wscale);
  CK(cudaMemcpyAsync(ns.ic.p, &ns.hic, sizeof(IterConsts), cudaMemcpyHostToDevice, s));
  LinearSolve out;
  if (f32) gmres<float>(x, ns, K32, jmode, krtol, ns.R1.p, out.iters, out.relres, rs, abstol);
  else gmres<double>(x, ns, K64, jmode, krtol, ns.R1.p, out.iters, out.relres, rs, abstol);
  check_gs_timeout(x, ns);
  return out;
}

// ------------------------------------------------------------------ time-marching driver kernels

// max over cells of (|V| + a) dt / lengthScale (update_time_step,
// time_step.cc:202-214) as an order key; dt_c = dt[c], or dt0 when dt is null
__global__ void k_max_cfl(DevCase cs, DevMesh m, const double *__restrict__ W, const double *__restrict__ dt, double dt0,
                          unsigned long long *__restrict__ key) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= m.nc) return;
  const int nt = m.nt;
  const double p = W[c], u = W[nt + c], v = W[2 * nt + c], w = W[3 * nt + c], T = W[4 * nt + c];
  const double a = sound(cs, p, T);
  const double d = dt ? dt[c] : dt0;
  atomicMax(key, okey((sqrt(u * u + v * v + w * w) + a) * d / m.c_len[c]));
}

__global__ void k_fill_value(int n, double *__restrict__ out, double v) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = v;
}

// W += dW (update_variables, ns.cc:338-396) with the per-block partial sums of
// dp^2/dt^2, |dV|^2/dt^2, dT^2/dt^2; err bit 8 on a NaN/Inf update
__global__ void k_update_res(int nc, double *__restrict__ Wn, const double *__restrict__ dW, const double *__restrict__ dt,
                             double *__restrict__ part, int *__restrict__ err) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  double r[3] = {0., 0., 0.};
  if (c < nc) {
    double d[5];
    bool bad = false;
    for (int k = 0; k < 5; ++k) {
      d[k] = dW[(size_t)k * nc + c];
      if (!isfinite(d[k])) bad = true;
    }
    if (bad) atomicOr(err, 8);
    for (int k = 0; k < 5; ++k) Wn[(size_t)k * nc + c] += d[k];
    const double dt2 = dt[c] * dt[c];
    r[0] = d[0] * d[0] / dt2;
    r[1] = d[1] * d[1] / dt2 + d[2] * d[2] / dt2 + d[3] * d[3] / dt2;
    r[2] = d[4] * d[4] / dt2;
  }
  __shared__ double sh[3][8];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int i = 0; i < 3; ++i) {
    double t = r[i];
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

// Boundary loads of the residual just evaluated (ns_assemble_linear_system.cc:
// 108-119): per listed BC j, force += F_conv - F_diff of the momentum
// equations (= -D), moment += (x_f - center) x force_f; per-block partial sums
// part[blk][j][6]
constexpr int kLoadBlock = 256;
__global__ void __launch_bounds__(kLoadBlock) k_loads_moment(DevMesh m, const double *__restrict__ D, int nlist,
                                                            const int *__restrict__ list, double cx, double cy, double cz,
                                                            double *__restrict__ part) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  __shared__ double sh[kMaxBC][6][kLoadBlock / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int j = -1;
  double F[3] = {0., 0., 0.}, M[3] = {0., 0., 0.};
  if (f < m.nf) {
    const int b = m.f_bc[f];
    for (int q = 0; q < nlist; ++q)
      if (list[q] == b) { j = q; break; }
    if (j >= 0) {
      for (int i = 0; i < 3; ++i) F[i] = -D[(size_t)(1 + i) * m.nf + f];
      const double r0 = m.f_x[f] - cx, r1 = m.f_x[m.nf + f] - cy, r2 = m.f_x[2 * m.nf + f] - cz;
      M[0] = r1 * F[2] - r2 * F[1];
      M[1] = r2 * F[0] - r0 * F[2];
      M[2] = r0 * F[1] - r1 * F[0];
    }
  }
  for (int q = 0; q < nlist; ++q)
    for (int i = 0; i < 6; ++i) {
      double t = (j == q) ? (i < 3 ? F[i] : M[i - 3]) : 0.;
      for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
      if (lane == 0) sh[q][i][wid] = t;
    }
  __syncthreads();
  if (threadIdx.x < nlist * 6) {
    const int q = threadIdx.x / 6, i = threadIdx.x % 6;
    double t = 0.;
    for (int k = 0; k < kLoadBlock / 32; ++k) t += sh[q][i][k];
    part[((size_t)blockIdx.x * nlist + q) * 6 + i] = t;
  }
}

void restart_write(const char *dir, int gid, int step, double time, const double *first_res, const double *rans_first,
                   int n_cells, int n_nodes, const double *W, const double *dt, const double *K, const double *mu_t);
void restart_read(const char *dir, int gid, int step, int n_cells, double *time, double *first_res, double *rans_first,
                  double *W, double *K, double *mu_t);

}  // namespace fcfd

using namespace fcfd;

extern "C" {

int fcfd_newton_solve(fcfd_ctx *x, double *W, const fcfd_newton_opts *o, fcfd_newton_report *rep) {
  try {
    if (!x || !W || !o || !rep) throw Error(FCFD_ERR_INPUT, "null argument");
    CK(cudaSetDevice(x->device));
    const DevMesh &m = x->dm;
    const int nc = m.nc, n = 5 * nc;
    cudaStream_t s = x->stream;
    const int tb = 256, gc = (nc + tb - 1) / tb, gn = (n + tb - 1) / tb;
    std::memset(rep, 0, sizeof(*rep));
    NewtonState ns;
    alloc_state(x, ns, o->precond_sweeps, o->krylov_cycles, o->fp32_krylov != 0, o->gs_launch, o->precond_ilu0 != 0);
    CK(cudaMemcpyAsync(x->Win.p, W, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    k_aos_to_soa_nc<<<gc, tb, 0, s>>>(x->Win.p, ns.Wn.p, nc);
    const int mdim = o->krylov_dim > 0 ? o->krylov_dim : 30;
    Krylov<double> K64;
    Krylov<float> K32;
    const bool f32 = o->fp32_krylov != 0;
    x->newton_frozen = o->jvp_mode == 1 || o->jvp_mode == 4;
    x->newton_f32 = o->jvp_mode == 3 || o->jvp_mode == 4;
    const int jmode = o->jvp_mode == 0 ? 0 : 1;
    if (f32) K32.alloc(x, mdim); else K64.alloc(x, mdim);
    DBuf<double> part, hh;
    part.alloc(kRedBlocks); hh.alloc(1);
    DBuf<double> Wsave;
    Wsave.alloc(n);
    DBuf<unsigned long long> key;
    key.alloc(1);
    CK(cudaStreamSynchronize(s));
    auto t0 = std::chrono::steady_clock::now();
    eval_residual<double>(x, ns.Wn.p, ns.R0.p, (const double *)nullptr, (const double *)nullptr);
    check_err(x);
    auto row_norms = [&](double out[5]) {
      for (int v = 0; v < 5; ++v) out[v] = dnorm(x, part, hh, ns.R0.p + (size_t)v * nc, nc);
    };
    double rows[5];
    row_norms(rows);
    const double r0 = rows[0];  // mass (continuity) row
    // momentum (x, y, z together) and energy rows for the all-rows stopping test
    auto mom = [](const double r[5]) { return std::sqrt(r[1] * r[1] + r[2] * r[2] + r[3] * r[3]); };
    const double m0 = mom(rows), e0 = rows[4];
    double rm = r0, rmom = m0, ren = e0;
    rep->seconds_to_tol = -1.;
    rep->res0 = r0;
    const double cfl0 = o->cfl0 > 0 ? o->cfl0 : 1.;
    const double growth = o->cfl_growth > 0 ? o->cfl_growth : 1.2;
    const double cflmax = o->cfl_max > 0 ? o->cfl_max : 1e6;
    double cfl = cfl0, cfl_prev = cfl0;
    int status = FCFD_ERR_NOT_CONVERGED;
    const int maxit = o->max_newton > 0 ? o->max_newton : 200;
    // explicit start-up through the initial transient (local time steps at
    // cfl0) until the mass residual has dropped by startup_drop
    bool startup_failed = false;
    if (o->startup_steps > 0) {
      const double drop = o->startup_drop > 0. ? o->startup_drop : 1e-3;
      int k = 0;
      for (; k < o->startup_steps && rm > drop * r0; ++k) {
        k_local_dt<double><<<gc, tb, 0, s>>>(x->cs, m, x->p64.W.p, ns.dt.p, cfl0, nullptr);
        k_explicit_update<<<gc, tb, 0, s>>>(x->cs, nc, ns.Wn.p, ns.R0.p, ns.vol.p, ns.dt.p, x->err.p);
        int h = 0;
        CK(cudaMemcpyAsync(&h, x->err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        if (h & 8) {
          CK(cudaMemsetAsync(x->err.p, 0, sizeof(int), s));
          startup_failed = true;
          break;
        }
        eval_residual<double>(x, ns.Wn.p, ns.R0.p, (const double *)nullptr, (const double *)nullptr);
        check_err(x);
        rm = dnorm(x, part, hh, ns.R0.p, nc);
        if (!std::isfinite(rm)) { startup_failed = true; break; }
      }
      rep->startup_steps = k;
      row_norms(rows);
      rmom = mom(rows);
      ren = rows[4];
    }
    const int hist = (int)(sizeof(rep->history) / sizeof(rep->history[0]));
    int rejects = 0;
    for (int it = 0; it < maxit && !startup_failed; ++it) {
      if (it < hist) {
        rep->history[it] = rm / r0;
        rep->seconds_history[it] = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
      }
      if (rm <= o->tol * r0) {
        if (rep->seconds_to_tol < 0.)
          rep->seconds_to_tol = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (!o->stop_all_rows || ((rmom <= o->tol * m0 || m0 == 0.) && (ren <= o->tol * e0 || e0 == 0.))) {
          status = FCFD_OK;
          break;
        }
      }
      if (o->max_seconds > 0 &&
          std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() > o->max_seconds) break;
      // local time step on the current state (loaded by the last residual)
      k_local_dt<double><<<gc, tb, 0, s>>>(x->cs, m, x->p64.W.p, ns.dt.p, cfl, nullptr);
      const double krtol = o->krylov_rtol > 0 ? o->krylov_rtol : 1e-2;
      const LinearSolve ls = implicit_solve(x, ns, K64, K32, f32, jmode, krtol, 0., part, hh);
      const int kit = ls.iters;
      rep->krylov_iterations += kit;
      // relax the update so that p and T change by at most 20 % per step:
      // one factor for the whole update, or per cell (local_relax)
      CK(cudaMemcpyAsync(Wsave.p, ns.Wn.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
      if (o->local_relax) {
        k_update_local<<<gc, tb, 0, s>>>(x->cs, nc, ns.Wn.p, ns.R1.p, x->err.p);
      } else {
        CK(cudaMemsetAsync(key.p, 0, sizeof(unsigned long long), s));
        k_max_rel_change<<<gc, tb, 0, s>>>(x->cs, nc, ns.Wn.p, ns.R1.p, key.p);
        unsigned long long kh = 0;
        CK(cudaMemcpyAsync(&kh, key.p, sizeof(kh), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        double dmax = 0.;
        {
          unsigned long long b = (kh >> 63) ? (kh & 0x7fffffffffffffffull) : ~kh;
          std::memcpy(&dmax, &b, sizeof(dmax));
        }
        const double alpha = (dmax > 0.2) ? 0.2 / dmax : 1.;
        k_update<double><<<gn, tb, 0, s>>>(n, ns.Wn.p, ns.R1.p, alpha, x->err.p);
      }
      int h = 0;
      CK(cudaMemcpyAsync(&h, x->err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
      CK(cudaStreamSynchronize(s));
      double rnew = NAN;
      if (!(h & 8)) {
        eval_residual<double>(x, ns.Wn.p, ns.R0.p, (const double *)nullptr, (const double *)nullptr);
        CK(cudaMemcpyAsync(&h, x->err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        row_norms(rows);
        rnew = rows[0];
      }
      if (h) CK(cudaMemsetAsync(x->err.p, 0, sizeof(int), s));
      rep->newton_iterations = it + 1;
      if (!std::isfinite(rnew) || (h & 8)) {
        // reject the step: restore the state, cut the CFL, re-evaluate
        if (++rejects > 12) { status = FCFD_ERR_DIVERGED; break; }
        CK(cudaMemcpyAsync(ns.Wn.p, Wsave.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
        eval_residual<double>(x, ns.Wn.p, ns.R0.p, (const double *)nullptr, (const double *)nullptr);
        row_norms(rows);
        cfl = std::max(cfl * 0.25, 1e-3);
        cfl_prev = cfl;
        continue;
      }
      rejects = 0;
      rm = rnew;
      rmom = mom(rows);
      ren = rows[4];
      rep->last_cfl = cfl;
      // next CFL: reference ramp, or switched evolution/relaxation on |R_mass|
      double next;
      if (o->cfl_mode == 1) next = cfl0 * std::pow(r0 / rm, o->ser_exponent > 0 ? o->ser_exponent : 1.);
      else next = cfl * growth;
      next = std::min(next, cfl_prev * 2.);
      cfl_prev = cfl;
      cfl = std::min(std::max(next, 1e-3), cflmax);
    }
    if (startup_failed) status = FCFD_ERR_DIVERGED;
    CK(cudaStreamSynchronize(s));
    rep->wall_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    rep->res_final = rm;
    rep->rows_final[0] = rm / r0;
    rep->rows_final[1] = m0 > 0. ? rmom / m0 : 0.;
    rep->rows_final[2] = e0 > 0. ? ren / e0 : 0.;
    rep->status = status;
    if (rep->newton_iterations < hist) rep->history[rep->newton_iterations] = rm / r0;
    k_soa_to_aos_nc<<<gc, tb, 0, s>>>(ns.Wn.p, x->Win.p, nc);
    CK(cudaMemcpyAsync(W, x->Win.p, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (status != FCFD_OK) {
      set_last_error(status == FCFD_ERR_DIVERGED ? "Newton iteration diverged (NaN/Inf update)" : "Newton iteration did not reach the tolerance");
      return status;
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

// Diagonal blocks V P/dt - J_cc of the implicit operator at the state W[nc][5]
// (host) and local time steps dt[nc] (host): the matrix the block
// preconditioner of fcfd_newton_solve / fcfd_run inverts, the counterpart of
// the diagonal of the matrix NavierStokes::time_terms (ns_time_terms.cc:
// 107-186, cons2prim 26-56) and assemble_linear_system's first-order Jacobian
// (ns_assemble_linear_system.cc:142-190) build.  blocks[nc][5][5] (row =
// equation, column = primitive variable).
int fcfd_time_terms(fcfd_ctx *x, const double *W, const double *dt, double *blocks) {
  try {
    if (!x || !W || !dt || !blocks) throw Error(FCFD_ERR_INPUT, "null argument");
    CK(cudaSetDevice(x->device));
    const DevMesh &m = x->dm;
    const int nc = m.nc, n = 5 * nc;
    cudaStream_t s = x->stream;
    const int tb = 256, gc = (nc + tb - 1) / tb;
    DBuf<double> Wn, dtd, B;
    Wn.alloc(n); dtd.alloc(nc); B.alloc(25 * (size_t)nc);
    CK(cudaMemcpyAsync(dtd.p, dt, sizeof(double) * nc, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(x->Win.p, W, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    k_aos_to_soa_nc<<<gc, tb, 0, s>>>(x->Win.p, Wn.p, nc);
    k_time_blocks<<<gc, tb, 0, s>>>(x->cs, nc, Wn.p, m.c_vol, dtd.p, B.p);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(blocks, B.p, sizeof(double) * 25 * (size_t)nc, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
  } catch (const Error &e) {
    set_last_error(e.what());
    return e.code;
  } catch (const std::exception &e) {
    set_last_error(e.what());
    return FCFD_ERR_INPUT;
  }
  return FCFD_OK;
}

int fcfd_diag_blocks(fcfd_ctx *x, const double *W, const double *dt, double *blocks) {
  try {
    if (!x || !W || !dt || !blocks) throw Error(FCFD_ERR_INPUT, "null argument");
    CK(cudaSetDevice(x->device));
    const DevMesh &m = x->dm;
    const int nc = m.nc, n = 5 * nc;
    cudaStream_t s = x->stream;
    const int tb = 256, gc = (nc + tb - 1) / tb;
    DBuf<double> Wn, R, dtd, vol, JL, JR, B;
    Wn.alloc(n); R.alloc(n); dtd.alloc(nc); vol.alloc(nc);
    JL.alloc(25 * (size_t)m.nf); JR.alloc(25 * (size_t)m.nf); B.alloc(25 * (size_t)nc);
    CK(cudaMemsetAsync(JR.p, 0, sizeof(double) * 25 * (size_t)m.nf, s));
    std::vector<double> hv(x->mesh->c_volume.begin(), x->mesh->c_volume.begin() + nc);
    CK(cudaMemcpyAsync(vol.p, hv.data(), sizeof(double) * nc, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(dtd.p, dt, sizeof(double) * nc, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(x->Win.p, W, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    k_aos_to_soa_nc<<<gc, tb, 0, s>>>(x->Win.p, Wn.p, nc);
    eval_residual<double>(x, Wn.p, R.p, (const double *)nullptr, (const double *)nullptr);
    launch_face_jac(x, JL.p, JR.p);
    k_diag_blocks<<<gc, tb, 0, s>>>(x->cs, m, Wn.p, vol.p, dtd.p, JL.p, JR.p, B.p);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(blocks, B.p, sizeof(double) * 25 * (size_t)nc, cudaMemcpyDeviceToHost, s));
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

// Deck-driven time loop (main.cc:294-438) for one laminar / Euler grid: per
// step update_time_step (time_step.cc:143-224: ramp, CFL schedule file, FIXED /
// CFL_MAX / CFL_LOCAL step, max CFL, physical time), one implicit
// backward-Euler step (NavierStokes::solve, ns.cc:104-118: residual, boundary
// loads, (V P/dt - J) dW = R by GMRES with the deck's relative / absolute
// tolerance and iteration cap, W += dW), the residual measure of
// update_variables (ns.cc:338-396), convergence.dat and screen lines
// (main.cc:351-369), loads files (write_loads, write_volume_output.cc:65-85),
// restart files (write_restart.cc:45-100; also when a file named dump_restart
// appears in the run directory), and every `updatefrequency` steps a re-read
// of the deck's timemarching section (update_time_step_options).
int fcfd_run(fcfd_ctx *x, double *W, const fcfd_run_opts *o, fcfd_run_report *rep) {
  try {
    if (!x || !W || !o || !rep) throw Error(FCFD_ERR_INPUT, "null argument");
    CK(cudaSetDevice(x->device));
    std::memset(rep, 0, sizeof(*rep));
    const fcfd_case &cs = *x->case_ptr;
    // turbulent decks: one coupled implicit solve per time step on (W, K)
    const bool turb = cs.turbulent;
    if (turb && !o->K) throw Error(FCFD_ERR_INPUT, "a turbulent deck needs opts->K (k and omega per cell, in/out)");
    TimeMarching tm = cs.tm;
    if (tm.ps_steps > 1) throw Error(FCFD_ERR_UNSUPPORTED, "pseudo-time (dual time stepping) iterations are not on the B200 path");
    if ((int)cs.load_bcs.size() > kMaxBC) throw Error(FCFD_ERR_UNSUPPORTED, "more than 16 load BCs");
    const DevMesh &m = x->dm;
    const int nc = m.nc, n = 5 * nc;
    cudaStream_t s = x->stream;
    const int tb = 256, gc = (nc + tb - 1) / tb;
    const std::string wd = (o->work_dir && *o->work_dir) ? std::string(o->work_dir) : std::string(".");
    auto in_dir = [&](const std::string &f) { return (!f.empty() && f[0] == '/') ? f : wd + "/" + f; };
    auto exists = [](const std::string &f) { std::ifstream t(f); return t.good(); };
    const int restart_step = o->restart_step > 0 ? o->restart_step : 0;
    double time = 0.;
    double first[3] = {0., 0., 0.};
    double first_rans[2] = {0., 0.};
    std::vector<double> mut_h(turb ? nc : 0);
    if (restart_step > 0)
      restart_read(wd.c_str(), 1, restart_step, nc, &time, first, first_rans, W, turb ? o->K : nullptr,
                   turb ? mut_h.data() : nullptr);
    // solver state (one GMRES cycle of at most `maximumiterations` vectors)
    NewtonState ns;
    alloc_state(x, ns, o->precond_sweeps, 1, o->fp32_krylov != 0);
    const int mdim = cs.lin_maxits > 0 ? cs.lin_maxits : 10;
    Krylov<double> K64;
    Krylov<float> K32;
    const bool f32 = o->fp32_krylov != 0;
    x->newton_frozen = o->jvp_mode == 1 || o->jvp_mode == 4;
    x->newton_f32 = o->jvp_mode == 3 || o->jvp_mode == 4;
    const int jmode = o->jvp_mode == 0 ? 0 : 1;
    if (f32) K32.alloc(x, mdim); else K64.alloc(x, mdim);
    struct KwGuard { void *p = nullptr; ~KwGuard() { if (p) kw_driver_destroy(p); } } kd;
    if (turb) kd.p = kw_driver_create(x, W, o->K, mdim);
    DBuf<double> part, hh, lpart, hdt;
    part.alloc(kRedBlocks); hh.alloc(1);
    DBuf<unsigned long long> key;
    key.alloc(1);
    DBuf<int> lbcs;
    const int nl = (int)cs.load_bcs.size();
    const int nlb = (m.nf + kLoadBlock - 1) / kLoadBlock;
    if (nl > 0) { lbcs.upload(cs.load_bcs); lpart.alloc((size_t)nlb * nl * 6); }
    DBuf<double> upart;
    upart.alloc((size_t)gc * (turb ? 5 : 3));
    CK(cudaMemcpyAsync(x->Win.p, W, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    k_aos_to_soa_nc<<<gc, tb, 0, s>>>(x->Win.p, ns.Wn.p, nc);
    // schedule file (set_time_step_options, time_step.cc:44-58)
    bool schedule = false;
    auto check_schedule = [&]() {
      schedule = false;
      if (!tm.schedule_file.empty()) {
        if (exists(in_dir(tm.schedule_file))) { tm.type = TS_CFL_MAX; schedule = true; }
        else if (o->echo) std::printf("[W] CFL schedule file %s is not found, continuing\n", tm.schedule_file.c_str());
      }
    };
    check_schedule();
    if (tm.type == TS_NONE) throw Error(FCFD_ERR_INPUT, "timemarching needs stepsize, CFLmax or CFLlocal");
    double cfl_max = tm.cfl_max, cfl_local = tm.cfl_local, ts_cur = tm.stepsize;
    double cfl_max_target = cfl_max, cfl_local_target = cfl_local, ts_target = ts_cur;
    bool ramp = tm.ramp;
    int n_steps = o->max_steps > 0 ? o->max_steps : tm.n_steps;
    int update_freq = tm.update_freq > 0 ? tm.update_freq : 1000000;
    const int load_freq = cs.load_freq > 0 ? cs.load_freq : 1000000;
    const int restart_freq = cs.restart_freq > 0 ? cs.restart_freq : 1000000;
    // convergence.dat (main.cc:302-305): appended to on a restart
    const std::string conv_name = wd + "/convergence.dat";
    FILE *conv = std::fopen(conv_name.c_str(), (restart_step > 0 && exists(conv_name)) ? "a" : "w");
    if (!conv) throw Error(FCFD_ERR_INPUT, "convergence.dat could not be opened in " + wd);
    struct Closer { FILE *f; ~Closer() { if (f) std::fclose(f); } } closer{conv};
    if (o->echo) {
      std::printf("[I] Beginning time loop\n\n");
      std::printf("=============================================================================================================\n");
      std::printf("step -- for each grid -> [grid-no  time  -- for each equation -> {cfl-max linear-iterations total-residual} ]\n");
      std::printf("=============================================================================================================\n");
    }
    if (nl > 0) mkdir((wd + "/volume_output").c_str(), S_IRWXU);
    std::vector<double> host_W(n), host_dt(nc), host_K(turb ? 2 * (size_t)nc : 0);
    auto save_restart = [&](int step) {
      if (turb) {
        // the eddy viscosity of the updated state, as RANS::solve leaves it
        // (update_eddy_viscosity after update_variables, rans.cc:85-98)
        kw_driver_residual(x, kd.p);
        kw_driver_state(x, kd.p, host_W.data(), host_K.data(), mut_h.data());
      } else {
        k_soa_to_aos_nc<<<gc, tb, 0, s>>>(ns.Wn.p, x->Win.p, nc);
        CK(cudaMemcpyAsync(host_W.data(), x->Win.p, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
      }
      CK(cudaMemcpyAsync(host_dt.data(), ns.dt.p, sizeof(double) * nc, cudaMemcpyDeviceToHost, s));
      CK(cudaStreamSynchronize(s));
      restart_write(wd.c_str(), 1, step, time, first, turb ? first_rans : nullptr, nc, (int)(x->mesh->nodes.size() / 3),
                    host_W.data(), host_dt.data(), turb ? host_K.data() : nullptr, turb ? mut_h.data() : nullptr);
    };
    auto t0 = std::chrono::steady_clock::now();
    int status = FCFD_OK;
    double res = 0.;
    for (int step = restart_step + 1; step <= n_steps + restart_step; ++step) {
      const bool last = step == n_steps + restart_step;
      // ---- update_time_step (time_step.cc:143-224)
      if (ramp) {
        if (step == 1) {
          if (tm.type == TS_FIXED) ts_cur = tm.ramp_initial;
          if (tm.type == TS_CFL_MAX) cfl_max = tm.ramp_initial;
          if (tm.type == TS_CFL_LOCAL) cfl_local = tm.ramp_initial;
        } else {
          if (tm.type == TS_FIXED) ts_cur = std::min(ts_cur * tm.ramp_growth, ts_target);
          if (tm.type == TS_CFL_MAX) cfl_max = std::min(cfl_max * tm.ramp_growth, cfl_max_target);
          if (tm.type == TS_CFL_LOCAL) cfl_local = std::min(cfl_local * tm.ramp_growth, cfl_local_target);
        }
      }
      // the state and its residual (the residual also loads W into the
      // gradient / limiter pipeline that the time step reads)
      if (turb) kw_driver_residual(x, kd.p);
      else eval_residual<double>(x, ns.Wn.p, ns.R0.p, (const double *)nullptr, (const double *)nullptr);
      double max_cfl = -1.;
      if (tm.type == TS_FIXED) {
        k_fill_value<<<gc, tb, 0, s>>>(nc, ns.dt.p, ts_cur);
      } else if (tm.type == TS_CFL_MAX) {
        if (schedule) {
          std::ifstream f(in_dir(tm.schedule_file));
          int st;
          double val;
          while (f >> st >> val) {
            if (step > st) { cfl_max = val; ramp = false; }
            else break;
          }
        }
        CK(cudaMemsetAsync(x->dtmin.p, 0xFF, sizeof(unsigned long long), s));
        k_local_dt<double><<<gc, tb, 0, s>>>(x->cs, m, x->p64.W.p, ns.dt.p, cfl_max, x->dtmin.p);
        k_fill_min<double><<<gc, tb, 0, s>>>(nc, ns.dt.p, x->dtmin.p);
        unsigned long long kmin = 0;
        CK(cudaMemcpyAsync(&kmin, x->dtmin.p, sizeof(kmin), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        unsigned long long b = (kmin >> 63) ? (kmin & 0x7fffffffffffffffull) : ~kmin;
        std::memcpy(&ts_cur, &b, sizeof(ts_cur));
      } else {
        CK(cudaMemsetAsync(x->dtmin.p, 0xFF, sizeof(unsigned long long), s));
        k_local_dt<double><<<gc, tb, 0, s>>>(x->cs, m, x->p64.W.p, ns.dt.p, cfl_local, x->dtmin.p);
      }
      if (tm.type == TS_CFL_LOCAL) {
        unsigned long long kmin = 0;
        CK(cudaMemcpyAsync(&kmin, x->dtmin.p, sizeof(kmin), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        unsigned long long b = (kmin >> 63) ? (kmin & 0x7fffffffffffffffull) : ~kmin;
        std::memcpy(&ts_cur, &b, sizeof(ts_cur));
        max_cfl = cfl_local;
      } else {
        CK(cudaMemsetAsync(key.p, 0, sizeof(unsigned long long), s));
        k_max_cfl<<<gc, tb, 0, s>>>(x->cs, m, x->p64.W.p, nullptr, ts_cur, key.p);
        unsigned long long kmax = 0;
        CK(cudaMemcpyAsync(&kmax, key.p, sizeof(kmax), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        unsigned long long b = (kmax >> 63) ? (kmax & 0x7fffffffffffffffull) : ~kmax;
        std::memcpy(&max_cfl, &b, sizeof(max_cfl));
      }
      time += ts_cur;
      // ---- boundary loads of this step's residual (before the Krylov solve
      // evaluates residuals at other states)
      std::vector<double> loads(6 * (size_t)nl, 0.);
      if (nl > 0 && step % load_freq == 0) {
        k_loads_moment<<<nlb, kLoadBlock, 0, s>>>(m, x->p64.D.p, nl, lbcs.p, cs.moment_center[0], cs.moment_center[1],
                                                  cs.moment_center[2], lpart.p);
        std::vector<double> hp((size_t)nlb * nl * 6);
        CK(cudaMemcpyAsync(hp.data(), lpart.p, sizeof(double) * hp.size(), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        for (int bl = 0; bl < nlb; ++bl)
          for (size_t k = 0; k < loads.size(); ++k) loads[k] += hp[(size_t)bl * nl * 6 + k];
      }
      // ---- implicit step
      LinearSolve ls;
      if (turb) ls.iters = kw_driver_step(x, kd.p, ns.dt.p, o->jvp_mode, cs.lin_rtol, cs.lin_abstol);
      else ls = implicit_solve(x, ns, K64, K32, f32, jmode, cs.lin_rtol, cs.lin_abstol, part, hh);
      rep->krylov_iterations += ls.iters;
      CK(cudaMemsetAsync(x->err.p, 0, sizeof(int), s));
      const int nsum = turb ? 5 : 3;
      if (turb) kw_driver_update(x, kd.p, ns.dt.p, upart.p, x->err.p);
      else k_update_res<<<gc, tb, 0, s>>>(nc, ns.Wn.p, ns.R1.p, ns.dt.p, upart.p, x->err.p);
      std::vector<double> hu((size_t)gc * nsum);
      int h = 0;
      CK(cudaMemcpyAsync(hu.data(), upart.p, sizeof(double) * hu.size(), cudaMemcpyDeviceToHost, s));
      CK(cudaMemcpyAsync(&h, x->err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
      CK(cudaStreamSynchronize(s));
      if (h & 8) {
        CK(cudaMemsetAsync(x->err.p, 0, sizeof(int), s));
        status = FCFD_ERR_DIVERGED;
        set_last_error("Divergence detected (NaN/Inf update) at time step " + std::to_string(step));
        rep->steps = step - restart_step;
        break;
      }
      double tot[5] = {0., 0., 0., 0., 0.};
      for (int bl = 0; bl < gc; ++bl)
        for (int i = 0; i < nsum; ++i) tot[i] += hu[(size_t)bl * nsum + i];
      if (step == 1) {
        for (int i = 0; i < 3; ++i) first[i] = std::sqrt(tot[i]);
        if (turb)
          for (int i = 0; i < 2; ++i) first_rans[i] = std::sqrt(tot[3 + i]);
      }
      res = 0.;
      for (int i = 0; i < 3; ++i) res += std::sqrt(tot[i]) / first[i] / 3.;
      // the k-omega residual of RANS::update_variables (rans.cc:240-250)
      double rres = 0.;
      if (turb)
        for (int i = 0; i < 2; ++i) rres += std::sqrt(tot[3 + i]) / first_rans[i] / 2.;
      // ---- screen and convergence.dat lines (main.cc:351-369; a turbulent
      // grid adds the k-omega solve's iterations and residual -- one coupled
      // solve here, so its iteration count is the flow's)
      char line[256];
      if (turb)
        std::snprintf(line, sizeof(line), "%d\t%d\t%.3e\t%.3e\t%d\t%.3e\t%d\t%.3e\n", step, 1, time, max_cfl, ls.iters, res,
                      ls.iters, rres);
      else
        std::snprintf(line, sizeof(line), "%d\t%d\t%.3e\t%.3e\t%d\t%.3e\n", step, 1, time, max_cfl, ls.iters, res);
      std::fputs(line, conv);
      std::fflush(conv);
      if (o->echo) std::fputs(line, stdout);
      rep->steps = step - restart_step;
      // ---- restart and loads files
      if (step % restart_freq == 0 || last) save_restart(step);
      if (nl > 0 && step % load_freq == 0) {
        for (int j = 0; j < nl; ++j) {
          const std::string fn = wd + "/volume_output/loads_grid_1_BC_" + std::to_string(cs.load_bcs[j] + 1) + ".dat";
          FILE *lf = std::fopen(fn.c_str(), "a");
          if (!lf) throw Error(FCFD_ERR_INPUT, "loads file " + fn + " could not be opened");
          const double *q = &loads[6 * (size_t)j];
          std::fprintf(lf, "%d\t%.8e\t%.8e\t%.8e\t%.8e\t%.8e\t%.8e\t%.8e\n", step, time, q[0], q[1], q[2], q[3], q[4], q[5]);
          std::fclose(lf);
        }
      }
      // ---- option re-read (main.cc:386-390)
      if (step % update_freq == 0) {
        tm = read_time_marching(cs.deck_path);
        check_schedule();
        cfl_max = cfl_max_target = tm.cfl_max;
        cfl_local = cfl_local_target = tm.cfl_local;
        ts_cur = ts_target = tm.stepsize;
        ramp = tm.ramp;
        update_freq = tm.update_freq > 0 ? tm.update_freq : 1000000;
        if (o->max_steps <= 0) n_steps = tm.n_steps;
      }
      if (exists(wd + "/dump_restart")) {
        save_restart(step);
        std::remove((wd + "/dump_restart").c_str());
      }
    }
    rep->wall_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    rep->time = time;
    rep->res = res;
    rep->status = status;
    if (turb) {
      kw_driver_state(x, kd.p, W, o->K, nullptr);
    } else {
      k_soa_to_aos_nc<<<gc, tb, 0, s>>>(ns.Wn.p, x->Win.p, nc);
      CK(cudaMemcpyAsync(W, x->Win.p, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
      CK(cudaStreamSynchronize(s));
    }
    if (o->echo) std::printf("[I] Wall time = %g second\n", rep->wall_seconds);
    return status;
  } catch (const Error &e) {
    set_last_error(e.what());
    return e.code;
  } catch (const std::exception &e) {
    set_last_error(e.what());
    return FCFD_ERR_INPUT;
  }
}

}  // extern "C"
