// k-omega RANS terms on the device, coupled to the NS residual through the
// eddy viscosity (rans_terms.cc:39-275, rans_update_eddy_viscosity.cc:26-56,
// rans_set_bcs.cc:25-83, rans.cc:27-71).
//
// One evaluation for the state (W, K = (k, omega)):
//   ghost update + extrema (NS) -> ghost k, omega and the eddy viscosity of
//   every cell -> its face values -> NS gradients + limiter -> outlet density
//   -> NS face flux with mu_t (also mdot and weightL per face) -> NS gather
//   -> LSQ gradients of k, omega -> k-omega face fluxes -> gather + sources.
// Ghost k, omega are the BC value where the reference fixes them on the BC
// (inlets) and the parent value otherwise: the RANS update_boundaries is
// missing from the reference snapshot and is reconstructed like the NS one.
#include <algorithm>
#include <cmath>
#include <vector>

#include "ctx.hpp"

namespace fcfd {

extern template __global__ void k_ghost_minmax<double>(DevCase, DevMesh, double *, unsigned long long *, int *);
extern template __global__ void k_ghost_minmax<Dual<double>>(DevCase, DevMesh, Dual<double> *, unsigned long long *, int *);
extern template __global__ void k_ghost_minmax<Dual<float>>(DevCase, DevMesh, Dual<float> *, unsigned long long *, int *);

// rans.cc:43-49, model=k-omega (blending = 1)
struct KOmega {
  static constexpr double sigma_k = 0.85, sigma_omega = 0.5, beta = 0.075, beta_star = 0.09, alpha = 5. / 9.;
};

// Per-state buffers of one coupled evaluation (S = double for the residual,
// Dual<double> for its tangent).
template <class S>
struct RansBuf {
  DBuf<S> K, GK, mut, mutf, DK, RK, mdot, wl;
  bool ready = false;
  void alloc(int nc, int nt, int nf) {
    K.alloc(2 * (size_t)nt); GK.alloc(6 * (size_t)nc); mut.alloc(nt); mutf.alloc(nf); DK.alloc(2 * (size_t)nf);
    RK.alloc(2 * (size_t)nc); mdot.alloc(nf); wl.alloc(nf);
    ready = true;
  }
};

struct RansState {
  RansBuf<double> b;
  RansBuf<Dual<double>> d;  // tangent buffers, allocated by the first fcfd_rans_jvp
  RansBuf<Dual<float>> f;   // the same for the FP32 tangent
  DBuf<double> vol;
};

void rans_free(fcfd_ctx *x) {
  delete x->rans;
  x->rans = nullptr;
}

namespace {

template <class S>
__device__ __forceinline__ S face_avg(const DevMesh &m, int f, const S *x) {
  return m.f_w[f] * x[m.f_parent[f]] + m.f_w[m.nf + f] * x[m.f_neighbor[f]];
}

// Ghost k, omega, then mu_t = min(ratio * mu, rho k / omega) for every cell.
template <class S>
__global__ void k_rans_prep(DevCase cs, DevMesh m, const S *__restrict__ W, S *__restrict__ K,
                            S *__restrict__ mut, double ratio_limit) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int nc = m.nc, nt = m.nt;
  if (i >= nt) return;
  if (i >= nc) {
    const int f = m.bface[i - nc], pa = m.f_parent[f];
    const DevBC &bc = cs.bc[m.f_bc[f]];
    if (bc.kw_fixed) { K[i] = S(bc.k_bc); K[nt + i] = S(bc.omega_bc); }
    else { K[i] = K[pa]; K[nt + i] = K[nt + pa]; }
  }
  const S p = W[i], T = W[4 * nt + i];
  const S rho = eos_rho(cs, p, T);
  const S mu = viscosity(cs, T);
  const S mt = rho * K[i] / K[nt + i];
  mut[i] = smin(S(ratio_limit * mu), mt);
}

// mu_t.face (variable.h:134-147): the BC value where fixed, else the average.
template <class S>
__global__ void k_rans_mutf(DevCase cs, DevMesh m, const S *__restrict__ mut, S *__restrict__ mutf) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= m.nf) return;
  const int b = m.f_bc[f];
  mutf[f] = (b >= 0 && cs.bc[b].mut_fixed) ? S(cs.bc[b].mut_bc) : face_avg(m, f, mut);
}

// LSQ gradients of k and omega (RANS::calc_cell_grads, rans.cc:167-173),
// the same weights as the flow gradients in their fused form.
template <class S>
__global__ void k_rans_grad(DevMesh m, const S *__restrict__ K, S *__restrict__ GK) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int nc = m.nc, nt = m.nt;
  if (c >= nc) return;
  const double xc0 = m.c_x[c], xc1 = m.c_x[nt + c], xc2 = m.c_x[2 * nt + c];
  const S u0[2] = {K[c], K[nt + c]};
  S acc[6] = {S(0.), S(0.), S(0.), S(0.), S(0.), S(0.)};
  for (int j = m.st_index[c]; j < m.st_index[c + 1]; ++j) {
    const int k = m.st_keys[j];
    if (k == c) continue;
    const double d0 = m.c_x[k] - xc0, d1 = m.c_x[nt + k] - xc1, d2 = m.c_x[2 * nt + k] - xc2;
    const double w = d0 * d0 + d1 * d1 + d2 * d2;
    for (int v = 0; v < 2; ++v) {
      const S a = w * (K[v * nt + k] - u0[v]);
      acc[3 * v] = acc[3 * v] + a * d0;
      acc[3 * v + 1] = acc[3 * v + 1] + a * d1;
      acc[3 * v + 2] = acc[3 * v + 2] + a * d2;
    }
  }
  const double C00 = m.st_cof[c], C01 = m.st_cof[nc + c], C02 = m.st_cof[2 * nc + c];
  const double C11 = m.st_cof[3 * nc + c], C12 = m.st_cof[4 * nc + c], C22 = m.st_cof[5 * nc + c];
  const double id = 1. / m.st_cof[6 * nc + c];
  const double M0 = m.st_mirror[c], M1 = m.st_mirror[nc + c], M2 = m.st_mirror[2 * nc + c];
  for (int v = 0; v < 2; ++v) {
    const S s0 = acc[3 * v], s1 = acc[3 * v + 1], s2 = acc[3 * v + 2];
    GK[(3 * v) * nc + c] = (C00 * s0 + C01 * s1 + C02 * s2) * id - M0 * u0[v];
    GK[(3 * v + 1) * nc + c] = (C01 * s0 + C11 * s1 + C12 * s2) * id - M1 * u0[v];
    GK[(3 * v + 2) * nc + c] = (C02 * s0 + C12 * s1 + C22 * s2) * id - M2 * u0[v];
  }
}

// k and omega face fluxes: DK = diffusive - convective (rans_terms.cc:59-112,
// get_kOmega 277-319).
template <class S>
__global__ void k_rans_face(DevCase cs, DevMesh m, const S *__restrict__ W, const S *__restrict__ K,
                            const S *__restrict__ GK, const S *__restrict__ mutf,
                            const S *__restrict__ mdot, const S *__restrict__ wl, S *__restrict__ DK) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  const int nf = m.nf, nc = m.nc, nt = m.nt;
  if (f >= nf) return;
  const int pa = m.f_parent[f], nb = m.f_neighbor[f], b = m.f_bc[f];
  const S Tf = (b >= 0 && cs.bc[b].T_fixed) ? S(cs.bc[b].T) : face_avg(m, f, W + 4 * nt);
  const S lam = viscosity(cs, Tf);
  const S turb = mutf[f];
  const S md = mdot[f], wL = wl[f], wR = 1. - wL;
  const S kL = K[pa], oL = K[nt + pa], kR = K[nb], oR = K[nt + nb];
  S gk[3], go[3];
  for (int i = 0; i < 3; ++i) {
    if (b >= 0) { gk[i] = GK[i * nc + pa]; go[i] = GK[(3 + i) * nc + pa]; }
    else {
      gk[i] = m.f_w[f] * GK[i * nc + pa] + m.f_w[nf + f] * GK[i * nc + nb];
      go[i] = m.f_w[f] * GK[(3 + i) * nc + pa] + m.f_w[nf + f] * GK[(3 + i) * nc + nb];
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
  DK[f] = diff0 - conv0;
  DK[nf + f] = diff1 - conv1;
}

// Per cell: sum of +-DK in ascending face order, plus sources x volume
// (rans_terms.cc:191-242).  RK is [nc][2].
template <class S>
__global__ void k_rans_gather(DevCase cs, DevMesh m, const S *__restrict__ W, const S *__restrict__ K,
                              const S *__restrict__ G, const S *__restrict__ mut,
                              const double *__restrict__ vol, const S *__restrict__ DK, S *__restrict__ RK) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int nc = m.nc, nt = m.nt, nf = m.nf;
  if (c >= nc) return;
  S r0 = S(0.), r1 = S(0.);
  for (int j = m.cf_index[c]; j < m.cf_index[c + 1]; ++j) {
    const int e = m.cf_list[j];
    if (e >= 0) { r0 = r0 + DK[e]; r1 = r1 + DK[nf + e]; }
    else { r0 = r0 + -1. * DK[~e]; r1 = r1 + -1. * DK[nf + ~e]; }
  }
  const S dudx = G[3 * nc + c], dudy = G[4 * nc + c], dudz = G[5 * nc + c];
  const S dvdx = G[6 * nc + c], dvdy = G[7 * nc + c], dvdz = G[8 * nc + c];
  const S dwdx = G[9 * nc + c], dwdy = G[10 * nc + c], dwdz = G[11 * nc + c];
  const S divU = dudx + dvdy + dwdz;
  const S sr = sqrt(2. * (dudx * dudx + dvdy * dvdy + dwdz * dwdz) + (dudy + dvdx) * (dudy + dvdx) +
                    (dudz + dwdx) * (dudz + dwdx) + (dvdz + dwdy) * (dvdz + dwdy));
  const S rho = eos_rho(cs, W[c], W[4 * nt + c]);
  const S k = K[c], om = K[nt + c], mt = mut[c];
  S Prod = mt * (sr * sr - 2. / 3. * divU * divU) - 2. / 3. * rho * k * divU;
  const S Dest = KOmega::beta_star * rho * om * k;
  Prod = smin(Prod, S(10. * Dest));
  const S s0 = Prod - Dest;
  const S s1 = KOmega::alpha * rho / mt * Prod - KOmega::beta * rho * om * om;
  RK[2 * c] = r0 + s0 * vol[c];
  RK[2 * c + 1] = r1 + s1 * vol[c];
}

__global__ void k_k_to_soa(const double *__restrict__ in, double *__restrict__ K, int nc, int nt) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  K[c] = in[2 * c];
  K[nt + c] = in[2 * c + 1];
}

// (value, tangent) AoS [nc][2] -> SoA duals with ghosts; duals -> AoS parts
template <class T>
__global__ void k_seed_kdual(const double *__restrict__ k, const double *__restrict__ dk, Dual<T> *__restrict__ K,
                             int nc, int nt) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  K[c] = Dual<T>(T(k[2 * c]), T(dk[2 * c]));
  K[nt + c] = Dual<T>(T(k[2 * c + 1]), T(dk[2 * c + 1]));
}
template <class T>
__global__ void k_split_kdual(const Dual<T> *__restrict__ RK, double *__restrict__ rk, double *__restrict__ drk, int nc) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  for (int v = 0; v < 2; ++v) {
    if (rk) rk[2 * c + v] = double(RK[2 * c + v].v);
    drk[2 * c + v] = double(RK[2 * c + v].d);
  }
}

double host_viscosity(const Material &mt, double T) {
  if (!mt.sutherland) return mt.mu;
  return mt.sut_mu_ref * std::pow((T + mt.Tref) / mt.sut_T_ref, 1.5) * (mt.sut_T_ref + mt.sut_S) / (T + mt.Tref + mt.sut_S);
}

}  // namespace

// RANS::set_bcs values: inlets fix k, omega and mu_t from the NS face values
// at initialisation (uniform IC state with the NS ghosts updated); no-slip
// walls fix mu_t = 0.  Runs the ghost kernel once on the IC state.
void rans_setup(fcfd_ctx *x) {
  const fcfd_case &c = *x->case_ptr;
  const fcfd_mesh &m = *x->mesh;
  if (!c.turbulent) return;
  if (!x->viscous) throw Error(FCFD_ERR_INPUT, "a turbulence model needs a viscous material");
  if (x->green_gauss) throw Error(FCFD_ERR_UNSUPPORTED, "the k-omega terms cover least-squares gradients only");
  const Material &mt = c.mat;
  const int nc = m.nc, nb = m.nb, nt = nc + nb, nf = m.nf;
  double p = c.ic_p, T = c.ic_T;
  const double R = mt.R;
  if (c.ic_has_p && c.ic_has_rho) T = (p + mt.Pref) / (R * c.ic_rho) - mt.Tref;
  else if (c.ic_has_rho && c.ic_has_T) p = c.ic_rho * R * (T + mt.Tref) - mt.Pref;
  std::vector<double> W(5 * (size_t)nt, 0.);
  for (int i = 0; i < nc; ++i) {
    W[i] = p; W[nt + i] = c.ic_V[0]; W[2 * (size_t)nt + i] = c.ic_V[1]; W[3 * (size_t)nt + i] = c.ic_V[2];
    W[4 * (size_t)nt + i] = T;
  }
  CK(cudaMemcpy(x->p64.W.p, W.data(), sizeof(double) * W.size(), cudaMemcpyHostToDevice));
  if (nb > 0) k_ghost_minmax<double><<<(nb + 255) / 256, 256, 0, x->stream>>>(x->cs, x->dm, x->p64.W.p, nullptr, x->err.p);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(x->stream));
  CK(cudaMemcpy(W.data(), x->p64.W.p, sizeof(double) * W.size(), cudaMemcpyDeviceToHost));
  auto rho_of = [&](double pp, double TT) { return (pp + mt.Pref) / (R * (TT + mt.Tref)); };
  for (size_t b = 0; b < c.bc.size(); ++b) {
    const BcRegion &r = c.bc[b];
    DevBC &o = x->cs.bc[b];
    o.kw_fixed = 0; o.mut_fixed = 0; o.k_bc = o.omega_bc = o.mut_bc = 0.;
    if (r.type == BC_INLET) {
      int fid = 0;
      for (int f = 0; f < nf; ++f)
        if (m.f_bc[f] == (int)b) { fid = f; break; }
      const int pa = m.f_parent[fid], g = m.f_neighbor[fid];
      const double w0 = m.f_w[2 * (size_t)fid], w1 = m.f_w[2 * (size_t)fid + 1];
      const bool here = m.f_bc[fid] == (int)b;
      const double rf = (r.rho_fixed && here) ? r.rho
                                              : w0 * rho_of(W[pa], W[4 * (size_t)nt + pa]) + w1 * rho_of(W[g], W[4 * (size_t)nt + g]);
      const double Tf = (r.T_fixed && here) ? r.T : w0 * W[4 * (size_t)nt + pa] + w1 * W[4 * (size_t)nt + g];
      double Vf[3];
      for (int k = 0; k < 3; ++k)
        Vf[k] = (r.V_fixed && here) ? r.V[k] : w0 * W[(1 + k) * (size_t)nt + pa] + w1 * W[(1 + k) * (size_t)nt + g];
      double kb = r.turb_intensity * std::sqrt(Vf[0] * Vf[0] + Vf[1] * Vf[1] + Vf[2] * Vf[2]);
      kb *= 1.5 * kb;
      kb = std::max(c.k_low, kb);
      o.kw_fixed = 1;
      o.k_bc = kb;
      o.omega_bc = rf * kb / (r.turb_ratio * host_viscosity(mt, Tf));
      o.mut_fixed = 1;
      o.mut_bc = r.turb_ratio * host_viscosity(mt, Tf);
    } else if (r.type == BC_WALL && r.kind != K_SLIP) {
      o.mut_fixed = 1;
      o.mut_bc = 0.;
    }
  }
  x->rans = new RansState();
  RansState &s = *x->rans;
  s.b.alloc(nc, nt, nf);
  std::vector<double> vol(m.c_volume.begin(), m.c_volume.begin() + nc);
  s.vol.upload(vol);
}

// One coupled evaluation; W and K already in P.W / s.K (interior parts).
// The NS residual goes to R (AoS [nc][5] when AOS, else SoA [5][nc]), the
// k-omega residual to RK (AoS [nc][2]).  With ev (3 events), ev[1] is
// recorded after the NS part (its gather) and ev[2] after the k-omega part.
// S = Dual<double> gives the tangent of both residuals (the tangent of the
// VK extrema through their first attaining cells, as in the NS chain).
template <class S, bool AOS>
static void rans_chain(fcfd_ctx *x, Pipe<S> &P, RansBuf<S> &s, S *mdot, S *wl, S *R, S *RK, cudaEvent_t *ev = nullptr) {
  const DevMesh &m = x->dm;
  cudaStream_t st = x->stream;
  const int tb = 256;
  const bool need_ext = x->cs.limiter == 1 && x->cs.order != 1;
  const int ng = (m.nb + tb - 1) / tb + (need_ext ? kExtremaBlocks : 0);
  if (ng > 0) k_ghost_minmax<S><<<ng, tb, 0, st>>>(x->cs, m, P.W.p, need_ext ? x->ext.p : nullptr, x->err.p);
  const int *argx = nullptr;
  if (!std::is_same<S, double>::value && need_ext) {
    k_argext<S><<<(m.nc + tb - 1) / tb, tb, 0, st>>>(m, P.W.p, x->ext.p, x->argx.p);
    argx = x->argx.p;
  }
  k_rans_prep<S><<<(m.nt + 127) / 128, 128, 0, st>>>(x->cs, m, P.W.p, s.K.p, s.mut.p, x->case_ptr->visc_ratio_limit);
  k_rans_mutf<S><<<(m.nf + 127) / 128, 128, 0, st>>>(x->cs, m, s.mut.p, s.mutf.p);
  launch_grad_limiter<S>(x->cs, m, P.W.p, x->ext.p, argx, P.G.p, P.Lm.p, st);
  launch_faces<S>(x, P, s.mutf.p, mdot, wl, st);
  k_gather<S, AOS><<<(5 * m.nc + tb - 1) / tb, tb, 0, st>>>(m, P.D.p, R, x->ext.p, x->argx.p);
  if (ev) CK(cudaEventRecord(ev[1], st));
  k_rans_grad<S><<<(m.nc + 127) / 128, 128, 0, st>>>(m, s.K.p, s.GK.p);
  k_rans_face<S><<<(m.nf + 127) / 128, 128, 0, st>>>(x->cs, m, P.W.p, s.K.p, s.GK.p, s.mutf.p, mdot, wl, s.DK.p);
  k_rans_gather<S><<<(m.nc + 127) / 128, 128, 0, st>>>(x->cs, m, P.W.p, s.K.p, P.G.p, s.mut.p, x->rans->vol.p, s.DK.p, RK);
  if (ev) CK(cudaEventRecord(ev[2], st));
  CK(cudaGetLastError());
}

}  // namespace fcfd

using namespace fcfd;

extern "C" int fcfd_rans_residual(fcfd_ctx *x, const double *W, const double *K, double *R, double *RK, int flags) {
  try {
    if (!x || !W || !K || !R || !RK) throw Error(FCFD_ERR_INPUT, "null argument");
    if (!x->rans) throw Error(FCFD_ERR_INPUT, "the case has no turbulence model");
    CK(cudaSetDevice(x->device));
    const DevMesh &m = x->dm;
    cudaStream_t s = x->stream;
    const bool dev = flags & FCFD_DEVICE_PTRS;
    const size_t n = 5 * (size_t)m.nc, nk = 2 * (size_t)m.nc;
    const double *w = W, *k = K;
    if (!dev) {
      CK(cudaMemcpyAsync(x->Win.p, W, sizeof(double) * n, cudaMemcpyHostToDevice, s));
      CK(cudaMemcpyAsync(x->rans->b.RK.p, K, sizeof(double) * nk, cudaMemcpyHostToDevice, s));
      w = x->Win.p;
      k = x->rans->b.RK.p;
    }
    const int tb = 256;
    k_aos_to_soa<double><<<(m.nc + tb - 1) / tb, tb, 0, s>>>(w, x->p64.W.p, m.nc, m.nt);
    k_k_to_soa<<<(m.nc + tb - 1) / tb, tb, 0, s>>>(k, x->rans->b.K.p, m.nc, m.nt);
    double *r = dev ? R : x->p64.R.p;
    double *rk = dev ? RK : x->rans->b.RK.p;
    rans_chain<double, true>(x, x->p64, x->rans->b, x->mdot.p, x->wl.p, r, rk);
    if (!dev) {
      CK(cudaMemcpyAsync(R, x->p64.R.p, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
      CK(cudaMemcpyAsync(RK, x->rans->b.RK.p, sizeof(double) * nk, cudaMemcpyDeviceToHost, s));
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

// Tangent of the coupled residual: (JV, JVK) = d(R, RK)/d(W, K) . (V, VK),
// evaluated by the same kernels on dual numbers; optionally (R, RK) too.
extern "C" int fcfd_rans_jvp(fcfd_ctx *x, const double *W, const double *K, const double *V, const double *VK,
                             double *R, double *RK, double *JV, double *JVK, int flags) {
  try {
    if (!x || !W || !K || !V || !VK || !JV || !JVK) throw Error(FCFD_ERR_INPUT, "null argument");
    if (!x->rans) throw Error(FCFD_ERR_INPUT, "the case has no turbulence model");
    if ((R == nullptr) != (RK == nullptr)) throw Error(FCFD_ERR_INPUT, "R and RK go together");
    CK(cudaSetDevice(x->device));
    const DevMesh &m = x->dm;
    cudaStream_t s = x->stream;
    const bool dev = flags & FCFD_DEVICE_PTRS;
    const size_t n = 5 * (size_t)m.nc, nk = 2 * (size_t)m.nc;
    const bool f32 = flags & FCFD_JVP_FP32;
    if (!f32 && !x->pjv.ready) x->pjv.alloc(m.nc, m.nf, m.nb);
    if (f32 && !x->pjv32.ready) x->pjv32.alloc(m.nc, m.nf, m.nb);
    RansBuf<Dual<double>> &d = x->rans->d;
    RansBuf<Dual<float>> &d32 = x->rans->f;
    if (!f32 && !d.ready) d.alloc(m.nc, m.nt, m.nf);
    if (f32 && !d32.ready) d32.alloc(m.nc, m.nt, m.nf);
    // host staging: W, V in Win / Vin; K, VK in the double k-omega buffers
    const double *w = W, *v = V, *k = K, *vk = VK;
    if (!dev) {
      CK(cudaMemcpyAsync(x->Win.p, W, sizeof(double) * n, cudaMemcpyHostToDevice, s));
      CK(cudaMemcpyAsync(x->Vin.p, V, sizeof(double) * n, cudaMemcpyHostToDevice, s));
      CK(cudaMemcpyAsync(x->rans->b.RK.p, K, sizeof(double) * nk, cudaMemcpyHostToDevice, s));
      CK(cudaMemcpyAsync(x->rans->b.DK.p, VK, sizeof(double) * nk, cudaMemcpyHostToDevice, s));
      w = x->Win.p; v = x->Vin.p; k = x->rans->b.RK.p; vk = x->rans->b.DK.p;
    }
    const int tb = 256;
    double *r = R ? (dev ? R : x->Rtmp.p) : nullptr;
    double *jv = dev ? JV : x->Vin.p;
    double *rk = R ? (dev ? RK : x->rans->b.RK.p) : nullptr;
    double *jk = dev ? JVK : x->rans->b.DK.p;
    if (f32) {
      k_seed_dual<float><<<(m.nc + tb - 1) / tb, tb, 0, s>>>(w, v, x->pjv32.W.p, m.nc, m.nt);
      k_seed_kdual<float><<<(m.nc + tb - 1) / tb, tb, 0, s>>>(k, vk, d32.K.p, m.nc, m.nt);
      rans_chain<Dual<float>, false>(x, x->pjv32, d32, d32.mdot.p, d32.wl.p, x->pjv32.R.p, d32.RK.p);
      k_split_dual<float><<<(m.nc + tb - 1) / tb, tb, 0, s>>>(x->pjv32.R.p, r, jv, m.nc);
      k_split_kdual<float><<<(m.nc + tb - 1) / tb, tb, 0, s>>>(d32.RK.p, rk, jk, m.nc);
    } else {
      k_seed_dual<double><<<(m.nc + tb - 1) / tb, tb, 0, s>>>(w, v, x->pjv.W.p, m.nc, m.nt);
      k_seed_kdual<double><<<(m.nc + tb - 1) / tb, tb, 0, s>>>(k, vk, d.K.p, m.nc, m.nt);
      rans_chain<Dual<double>, false>(x, x->pjv, d, d.mdot.p, d.wl.p, x->pjv.R.p, d.RK.p);
      k_split_dual<double><<<(m.nc + tb - 1) / tb, tb, 0, s>>>(x->pjv.R.p, r, jv, m.nc);
      k_split_kdual<double><<<(m.nc + tb - 1) / tb, tb, 0, s>>>(d.RK.p, rk, jk, m.nc);
    }
    CK(cudaGetLastError());
    if (!dev) {
      if (R) {
        CK(cudaMemcpyAsync(R, x->Rtmp.p, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(RK, x->rans->b.RK.p, sizeof(double) * nk, cudaMemcpyDeviceToHost, s));
      }
      CK(cudaMemcpyAsync(JV, x->Vin.p, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
      CK(cudaMemcpyAsync(JVK, x->rans->b.DK.p, sizeof(double) * nk, cudaMemcpyDeviceToHost, s));
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

// Device time of the coupled NS + k-omega residual on the state last passed
// to fcfd_rans_residual: out[0] total ms per evaluation, out[1] the NS part
// (with the eddy viscosity), out[2] the k-omega part; L2 flushed before each
// evaluation when flush_l2 is set.
extern "C" int fcfd_time_rans(fcfd_ctx *x, int reps, int flush_l2, double *out, int out_len) {
  try {
    if (!x || !out || reps < 1) throw Error(FCFD_ERR_INPUT, "bad argument");
    if (!x->rans) throw Error(FCFD_ERR_INPUT, "the case has no turbulence model");
    CK(cudaSetDevice(x->device));
    cudaStream_t s = x->stream;
    if (flush_l2 && x->flush.n == 0) x->flush.alloc((size_t)512 << 20);
    Timing t;
    double acc[3] = {0., 0., 0.};
    for (int r = 0; r < reps; ++r) {
      if (flush_l2) CK(cudaMemsetAsync(x->flush.p, r & 0xff, x->flush.n, s));
      CK(cudaEventRecord(t.ev[0], s));
      rans_chain<double, true>(x, x->p64, x->rans->b, x->mdot.p, x->wl.p, x->p64.R.p, x->rans->b.RK.p, t.ev);
      CK(cudaEventSynchronize(t.ev[2]));
      float ms;
      CK(cudaEventElapsedTime(&ms, t.ev[0], t.ev[2])); acc[0] += ms;
      CK(cudaEventElapsedTime(&ms, t.ev[0], t.ev[1])); acc[1] += ms;
      CK(cudaEventElapsedTime(&ms, t.ev[1], t.ev[2])); acc[2] += ms;
    }
    for (int k = 0; k < 3 && k < out_len; ++k) out[k] = acc[k] / reps;
  } catch (const Error &e) {
    set_last_error(e.what());
    return e.code;
  } catch (const std::exception &e) {
    set_last_error(e.what());
    return FCFD_ERR_INPUT;
  }
  return FCFD_OK;
}

extern "C" int fcfd_rans_bcs(const fcfd_ctx *x, double *out, int32_t out_len) {
  if (!x || !out) { set_last_error("null argument"); return FCFD_ERR_INPUT; }
  const int nbc = x->cs.nbc;
  if (out_len < 5 * nbc) { set_last_error("output too small"); return FCFD_ERR_INPUT; }
  for (int b = 0; b < nbc; ++b) {
    const DevBC &o = x->cs.bc[b];
    out[5 * b] = o.kw_fixed; out[5 * b + 1] = o.k_bc; out[5 * b + 2] = o.omega_bc;
    out[5 * b + 3] = o.mut_fixed; out[5 * b + 4] = o.mut_bc;
  }
  return FCFD_OK;
}
