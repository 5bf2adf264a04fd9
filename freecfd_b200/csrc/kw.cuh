// k-omega expressions shared by the coupled residual (rans.cu) and its
// adjoint (adjoint.cu): the eddy viscosity, the k / omega face flux and the
// cell sources, written once over a scalar type S (double, Dual<T>, DN<L>)
// so that the adjoint differentiates exactly the operations the residual
// performs.
#pragma once

#include "kernels.cuh"

namespace fcfd {

// rans.cc:43-49, model=k-omega (blending = 1)
struct KOmega {
  static constexpr double sigma_k = 0.85, sigma_omega = 0.5, beta = 0.075, beta_star = 0.09, alpha = 5. / 9.;
};

// mu_t = min(ratio * mu(T), rho k / omega) (rans_update_eddy_viscosity.cc:26-56)
template <class S>
__device__ __forceinline__ S kw_mut(const DevCase &cs, const S &p, const S &T, const S &k, const S &om, double ratio) {
  const S rho = eos_rho(cs, p, T);
  const S mu = viscosity(cs, T);
  const S mt = rho * k / om;
  return smin(S(ratio * mu), mt);
}

// k and omega face fluxes DK = diffusive - convective (rans_terms.cc:59-112,
// get_kOmega 277-319).  Tpa / Tnb: the cells' temperatures (the face value is
// their weighted average unless the BC fixes T); (kL, oL), (kR, oR): k and
// omega of the parent and the neighbour (ghost on a boundary face); gpa, gnb:
// the cells' k and omega gradients (gnb read on interior faces only); turb:
// the face eddy viscosity; md, wL: the NS face's mass flux and left weight.
template <class S>
__device__ __forceinline__ void kw_face_flux(const DevCase &cs, const DevMesh &m, int f, int b, int pa, int nb, const S &Tpa,
                                             const S &Tnb, const S &kL, const S &oL, const S &kR, const S &oR,
                                             const S gpa[6], const S gnb[6], const S &turb, const S &md, const S &wL,
                                             S &DK0, S &DK1) {
  const int nf = m.nf, nt = m.nt;
  const S Tf = (b >= 0 && cs.bc[b].T_fixed) ? S(cs.bc[b].T) : m.f_w[f] * Tpa + m.f_w[nf + f] * Tnb;
  const S lam = viscosity(cs, Tf);
  const S wR = 1. - wL;
  S gk[3], go[3];
  for (int i = 0; i < 3; ++i) {
    if (b >= 0) { gk[i] = gpa[i]; go[i] = gpa[3 + i]; }
    else {
      gk[i] = m.f_w[f] * gpa[i] + m.f_w[nf + f] * gnb[i];
      go[i] = m.f_w[f] * gpa[3 + i] + m.f_w[nf + f] * gnb[3 + i];
    }
  }
  const double l0 = m.c_x[nb] - m.c_x[pa], l1 = m.c_x[nt + nb] - m.c_x[nt + pa], l2 = m.c_x[2 * nt + nb] - m.c_x[2 * nt + pa];
  const double lm = sqrt(l0 * l0 + l1 * l1 + l2 * l2);
  const double e[3] = {l0 / lm, l1 / lm, l2 / lm};
  const S dk = gk[0] * e[0] + gk[1] * e[1] + gk[2] * e[2];
  const S dw = go[0] * e[0] + go[1] * e[1] + go[2] * e[2];
  for (int i = 0; i < 3; ++i) {
    gk[i] = gk[i] - dk * e[i] + (kR - kL) / lm * e[i];
    go[i] = go[i] - dw * e[i] + (oR - oL) / lm * e[i];
  }
  const double n[3] = {m.f_n[f], m.f_n[nf + f], m.f_n[2 * nf + f]};
  const double A = m.f_area[f];
  const S conv0 = md * (wL * kL + wR * kR) * A, conv1 = md * (wL * oL + wR * oR) * A;
  const S diff0 = (lam + turb * KOmega::sigma_k) * (gk[0] * n[0] + gk[1] * n[1] + gk[2] * n[2]) * A;
  const S diff1 = (lam + turb * KOmega::sigma_omega) * (go[0] * n[0] + go[1] * n[1] + go[2] * n[2]) * A;
  DK0 = diff0 - conv0;
  DK1 = diff1 - conv1;
}

// k and omega sources of a cell (rans_terms.cc:191-242) from its velocity
// gradient rows g9 = (du/dx, du/dy, du/dz, dv/dx, ..., dw/dz), its p, T, k,
// omega and eddy viscosity.
template <class S>
__device__ __forceinline__ void kw_source(const DevCase &cs, const S g9[9], const S &p, const S &T, const S &k, const S &om,
                                          const S &mt, S &s0, S &s1) {
  const S &dudx = g9[0], &dudy = g9[1], &dudz = g9[2];
  const S &dvdx = g9[3], &dvdy = g9[4], &dvdz = g9[5];
  const S &dwdx = g9[6], &dwdy = g9[7], &dwdz = g9[8];
  const S divU = dudx + dvdy + dwdz;
  const S sr = sqrt(2. * (dudx * dudx + dvdy * dvdy + dwdz * dwdz) + (dudy + dvdx) * (dudy + dvdx) +
                    (dudz + dwdx) * (dudz + dwdx) + (dvdz + dwdy) * (dvdz + dwdy));
  const S rho = eos_rho(cs, p, T);
  S Prod = mt * (sr * sr - 2. / 3. * divU * divU) - 2. / 3. * rho * k * divU;
  const S Dest = KOmega::beta_star * rho * om * k;
  Prod = smin(Prod, S(10. * Dest));
  s0 = Prod - Dest;
  s1 = KOmega::alpha * rho / mt * Prod - KOmega::beta * rho * om * om;
}

}  // namespace fcfd
