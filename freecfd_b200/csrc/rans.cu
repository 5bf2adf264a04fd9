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
#include <chrono>
#include <cmath>
#include <cstring>
#include <vector>

#include <limits>
#include <memory>

#include "ctx.hpp"
#include "kw.cuh"

namespace fcfd {

extern template __global__ void k_ghost_minmax<double>(DevCase, DevMesh, double *, unsigned long long *, int *);
extern template __global__ void k_ghost_minmax<Dual<double>>(DevCase, DevMesh, Dual<double> *, unsigned long long *, int *);
extern template __global__ void k_ghost_minmax<Dual<float>>(DevCase, DevMesh, Dual<float> *, unsigned long long *, int *);

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
  pdl_wait();
  pdl_trigger();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int nc = m.nc, nt = m.nt;
  if (i >= nt) return;
  if (i >= nc) {
    const int f = m.bface[i - nc], pa = m.f_parent[f];
    const DevBC &bc = cs.bc[m.f_bc[f]];
    if (bc.kw_fixed) { K[i] = S(bc.k_bc); K[nt + i] = S(bc.omega_bc); }
    else { K[i] = K[pa]; K[nt + i] = K[nt + pa]; }
  }
  mut[i] = kw_mut(cs, W[i], W[4 * nt + i], K[i], K[nt + i], ratio_limit);
}

// mu_t.face (variable.h:134-147): the BC value where fixed, else the average.
template <class S>
__global__ void k_rans_mutf(DevCase cs, DevMesh m, const S *__restrict__ mut, S *__restrict__ mutf) {
  pdl_wait();
  pdl_trigger();
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= m.nf) return;
  const int b = m.f_bc[f];
  mutf[f] = (b >= 0 && cs.bc[b].mut_fixed) ? S(cs.bc[b].mut_bc) : face_avg(m, f, mut);
}

// LSQ gradients of k and omega (RANS::calc_cell_grads, rans.cc:167-173),
// the same weights as the flow gradients in their fused form.
template <class S>
__global__ void k_rans_grad(DevMesh m, const S *__restrict__ K, S *__restrict__ GK) {
  pdl_wait();
  pdl_trigger();
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int nc = m.nc, nt = m.nt;
  if (c >= nc) return;
  if (m.st_w) {
    // stored map weights (curvilinear cases): grad += weight * phi in key order
    S g[6] = {S(0.), S(0.), S(0.), S(0.), S(0.), S(0.)};
    for (int j = m.st_index[c]; j < m.st_index[c + 1]; ++j) {
      const int k = m.st_keys[j];
      const double w0 = m.st_w[3 * (size_t)j], w1 = m.st_w[3 * (size_t)j + 1], w2 = m.st_w[3 * (size_t)j + 2];
      for (int v = 0; v < 2; ++v) {
        const S phi = K[v * nt + k];
        g[3 * v] = g[3 * v] + w0 * phi;
        g[3 * v + 1] = g[3 * v + 1] + w1 * phi;
        g[3 * v + 2] = g[3 * v + 2] + w2 * phi;
      }
    }
    for (int i = 0; i < 6; ++i) GK[i * nc + c] = g[i];
    return;
  }
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

// k and omega face fluxes: DK = diffusive - convective (kw_face_flux).
template <class S>
__global__ void k_rans_face(DevCase cs, DevMesh m, const S *__restrict__ W, const S *__restrict__ K,
                            const S *__restrict__ GK, const S *__restrict__ mutf,
                            const S *__restrict__ mdot, const S *__restrict__ wl, S *__restrict__ DK) {
  pdl_wait();
  pdl_trigger();
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  const int nf = m.nf, nc = m.nc, nt = m.nt;
  if (f >= nf) return;
  const int pa = m.f_parent[f], nb = m.f_neighbor[f], b = m.f_bc[f];
  S gpa[6], gnb[6];
  for (int i = 0; i < 6; ++i) {
    gpa[i] = GK[i * nc + pa];
    gnb[i] = b < 0 ? GK[i * nc + nb] : S(0.);
  }
  S d0, d1;
  kw_face_flux<S>(cs, m, f, b, pa, nb, W[4 * nt + pa], W[4 * nt + nb], K[pa], K[nt + pa], K[nb], K[nt + nb], gpa, gnb,
                  mutf[f], mdot[f], wl[f], d0, d1);
  DK[f] = d0;
  DK[nf + f] = d1;
}

// Per cell: sum of +-DK in ascending face order, plus sources x volume
// (rans_terms.cc:191-242).  RK is [nc][2].
template <class S>
__global__ void k_rans_gather(DevCase cs, DevMesh m, const S *__restrict__ W, const S *__restrict__ K,
                              const S *__restrict__ G, const S *__restrict__ mut,
                              const double *__restrict__ vol, const S *__restrict__ DK, S *__restrict__ RK) {
  pdl_wait();
  pdl_trigger();
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int nc = m.nc, nt = m.nt, nf = m.nf;
  if (c >= nc) return;
  S r0 = S(0.), r1 = S(0.);
  for (int j = m.cf_index[c]; j < m.cf_index[c + 1]; ++j) {
    const int e = m.cf_list[j];
    if (e >= 0) { r0 = r0 + DK[e]; r1 = r1 + DK[nf + e]; }
    else { r0 = r0 + -1. * DK[~e]; r1 = r1 + -1. * DK[nf + ~e]; }
  }
  S g9[9];
  for (int i = 0; i < 9; ++i) g9[i] = G[(3 + i) * nc + c];
  S s0, s1;
  kw_source<S>(cs, g9, W[c], W[4 * nt + c], K[c], K[nt + c], mut[c], s0, s1);
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
  const bool pdl = x->pdl;
  launch_k(pdl, k_rans_prep<S>, (m.nt + 127) / 128, 128, 0, st, x->cs, m, (const S *)P.W.p, s.K.p, s.mut.p,
           x->case_ptr->visc_ratio_limit);
  launch_k(pdl, k_rans_mutf<S>, (m.nf + 127) / 128, 128, 0, st, x->cs, m, (const S *)s.mut.p, s.mutf.p);
  launch_grad_limiter<S>(x->cs, m, P.W.p, x->ext.p, argx, P.G.p, P.Lm.p, st, pdl);
  launch_faces<S>(x, P, s.mutf.p, mdot, wl, st);
  k_gather<S, AOS><<<(5 * m.nc + tb - 1) / tb, tb, 0, st>>>(m, P.D.p, R, x->ext.p, x->argx.p);
  if (ev) CK(cudaEventRecord(ev[1], st));
  launch_k(pdl, k_rans_grad<S>, (m.nc + 127) / 128, 128, 0, st, m, (const S *)s.K.p, s.GK.p);
  launch_k(pdl, k_rans_face<S>, (m.nf + 127) / 128, 128, 0, st, x->cs, m, (const S *)P.W.p, (const S *)s.K.p,
           (const S *)s.GK.p, (const S *)s.mutf.p, (const S *)mdot, (const S *)wl, s.DK.p);
  launch_k(pdl, k_rans_gather<S>, (m.nc + 127) / 128, 128, 0, st, x->cs, m, (const S *)P.W.p, (const S *)s.K.p,
           (const S *)P.G.p, (const S *)s.mut.p, (const double *)x->rans->vol.p, (const S *)s.DK.p, RK);
  if (ev) CK(cudaEventRecord(ev[2], st));
  CK(cudaGetLastError());
}

void rans_eval_for_adjoint(fcfd_ctx *x, const double *W, const double *K, RansFwd &out) {
  const DevMesh &m = x->dm;
  cudaStream_t s = x->stream;
  RansBuf<double> &b = x->rans->b;
  const int tb = 256;
  k_aos_to_soa<double><<<(m.nc + tb - 1) / tb, tb, 0, s>>>(W, x->p64.W.p, m.nc, m.nt);
  k_k_to_soa<<<(m.nc + tb - 1) / tb, tb, 0, s>>>(K, b.K.p, m.nc, m.nt);
  rans_chain<double, false>(x, x->p64, b, x->mdot.p, x->wl.p, x->p64.R.p, b.RK.p);
  out.K = b.K.p; out.GK = b.GK.p; out.mut = b.mut.p; out.mutf = b.mutf.p;
  out.mdot = x->mdot.p; out.wl = x->wl.p; out.vol = x->rans->vol.p;
  out.ratio = x->case_ptr->visc_ratio_limit;
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

// ------------------------------------------------------------------ coupled k-omega Newton-Krylov
//
// Steady solve of the coupled flow + k-omega residual F(X) = (R(W, K), RK(W, K))
// by pseudo-transient Newton-Krylov: (D - dF/dX) dX = F(X), X += alpha dX,
// with D the time terms (V P/dt for the flow equations, ns_time_terms.cc:
// 107-186; rho V/dt on both k-omega rows, rans_time_terms.cc:25-87) and the
// local time step of the flow (time_step.cc:143-224).  The reference solves
// the two systems one after the other (NavierStokes::solve then RANS::solve,
// ns.cc:104-118, rans.cc:85-98); here they are one Newton system on
// X = [p u v w T k omega] (SoA [7][nc]).  J.v: a finite difference of the
// FP64 coupled residual, or the coupled tangent chain in FP32 (the mixed
// arm).  Preconditioner: block Jacobi, the flow blocks from the first-order
// face Jacobians with the face eddy viscosities (newton.cu), the k and omega
// rows by a diagonal of the time term, the first-order upwind convection and
// diffusion across the cell's faces and the destruction terms' derivatives.
// GMRES(m), right preconditioned, FP64 classical Gram-Schmidt twice, each
// equation weighted by the inverse of its initial residual norm.
namespace fcfd {
namespace kwn {

constexpr int kNv = 7;
constexpr int kRedBlk = 592;  // 4 x 148 blocks for the reductions

// X (SoA [7][nc]) + eps z -> the chain's W [5][nt] and K [2][nt] (interiors)
struct Wt7 {
  double s[kNv];
};
// per linear step constants the captured Arnoldi steps read from the device:
// equation weights, their inverses, the finite-difference numerator
struct KwIter {
  Wt7 wr, iwr;
  double eps_num;
};
// finite-difference step of the Krylov matvec, eps_num / |z| with |z|^2 read
// from the device (1e-8 where |z| = 0)
__device__ __forceinline__ double kw_fd_eps(double eps_num, const double *zz) {
  const double q = *zz;
  return q > 0. ? eps_num / sqrt(q) : 1e-8;
}
__global__ void k_x_load(int nc, int nt, const double *__restrict__ X, const double *__restrict__ z, double eps,
                         double *__restrict__ W, double *__restrict__ K, const KwIter *__restrict__ it = nullptr,
                         const double *__restrict__ zz = nullptr) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  if (zz) eps = kw_fd_eps(it->eps_num, zz);
#pragma unroll
  for (int v = 0; v < 5; ++v) W[v * nt + c] = X[v * nc + c] + (z ? eps * z[v * nc + c] : 0.);
#pragma unroll
  for (int v = 0; v < 2; ++v) K[v * nt + c] = X[(5 + v) * nc + c] + (z ? eps * z[(5 + v) * nc + c] : 0.);
}

// X and the direction z as FP32 duals of the tangent chain
__global__ void k_x_load_dual(int nc, int nt, const double *__restrict__ X, const double *__restrict__ z,
                              Dual<float> *__restrict__ W, Dual<float> *__restrict__ K) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
#pragma unroll
  for (int v = 0; v < 5; ++v) W[v * nt + c] = Dual<float>(float(X[v * nc + c]), float(z[v * nc + c]));
#pragma unroll
  for (int v = 0; v < 2; ++v) K[v * nt + c] = Dual<float>(float(X[(5 + v) * nc + c]), float(z[(5 + v) * nc + c]));
}

// k-omega residual AoS [nc][2] -> planes 5, 6 of F
__global__ void k_rk_planes(int nc, const double *__restrict__ RK, double *__restrict__ F) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  F[5 * nc + c] = RK[2 * c];
  F[6 * nc + c] = RK[2 * c + 1];
}

// tangent parts of the FP32 chain's outputs -> Jz [7][nc]
__global__ void k_dual_planes(int nc, const Dual<float> *__restrict__ R, const Dual<float> *__restrict__ RK,
                              double *__restrict__ Jz) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
#pragma unroll
  for (int v = 0; v < 5; ++v) Jz[v * nc + c] = double(R[v * nc + c].d);
  Jz[5 * nc + c] = double(RK[2 * c].d);
  Jz[6 * nc + c] = double(RK[2 * c + 1].d);
}

// y = wr * (D z - Jz): D the time terms; Jz = (F1 - F0) * inv_eps, or the
// tangent (F0 null).  wr: per-equation weights.
__global__ void k_kw_matvec(DevCase cs, int nc, const double *__restrict__ X, const double *__restrict__ vol,
                            const double *__restrict__ dt, const double *__restrict__ z, const double *__restrict__ F1,
                            const double *__restrict__ F0, double inv_eps, const KwIter *__restrict__ it,
                            double *__restrict__ y, const double *__restrict__ zz = nullptr) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  if (zz) inv_eps = 1. / kw_fd_eps(it->eps_num, zz);
  const Wt7 &wr = it->wr;
  const double p = X[c], u = X[nc + c], v = X[2 * nc + c], w = X[3 * nc + c], T = X[4 * nc + c];
  const double pressure = p + cs.Pref, temperature = T + cs.Tref;
  const double rho = pressure / (cs.R * temperature);
  const double drho_dT = -1. * rho / temperature, drho_dp = rho / pressure;
  const double H = cs.Cp * temperature + 0.5 * (u * u + v * v + w * w);
  const double s = vol[c] / dt[c];
  double zv[kNv];
#pragma unroll
  for (int k = 0; k < kNv; ++k) zv[k] = z[k * nc + c];
  double Dz[kNv];
  Dz[0] = s * (drho_dp * zv[0] + drho_dT * zv[4]);
  Dz[1] = s * (drho_dp * u * zv[0] + rho * zv[1] + drho_dT * u * zv[4]);
  Dz[2] = s * (drho_dp * v * zv[0] + rho * zv[2] + drho_dT * v * zv[4]);
  Dz[3] = s * (drho_dp * w * zv[0] + rho * zv[3] + drho_dT * w * zv[4]);
  Dz[4] = s * ((drho_dp * H - 1.) * zv[0] + rho * u * zv[1] + rho * v * zv[2] + rho * w * zv[3] +
               (drho_dT * H + rho * cs.Cp) * zv[4]);
  Dz[5] = s * rho * zv[5];
  Dz[6] = s * rho * zv[6];
#pragma unroll
  for (int k = 0; k < kNv; ++k) {
    const double jz = F0 ? (F1[k * nc + c] - F0[k * nc + c]) * inv_eps : F1[k * nc + c];
    y[k * nc + c] = wr.s[k] * (Dz[k] - jz);
  }
}

// Diagonal of the k and omega rows: rho V/dt, the outflow and diffusion
// coefficients over the cell's faces (first-order upwind convection with the
// faces' mass fluxes, (mu + sigma mu_t) A / |l2r|) and the derivatives of
// the destruction terms (beta* rho omega for k, 2 beta rho omega for omega).
__global__ void k_kw_diag(DevCase cs, DevMesh m, const double *__restrict__ X, const double *__restrict__ vol,
                          const double *__restrict__ dt, const double *__restrict__ mdot, const double *__restrict__ mutf,
                          double *__restrict__ dk) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int nc = m.nc, nt = m.nt, nf = m.nf;
  if (c >= nc) return;
  const double p = X[c], T = X[4 * nc + c], om = X[6 * nc + c];
  const double rho = (p + cs.Pref) / (cs.R * (T + cs.Tref));
  const double mu = viscosity(cs, T);
  double conv = 0., dk0 = 0., dk1 = 0.;
  for (int j = m.cf_index[c]; j < m.cf_index[c + 1]; ++j) {
    const int e = m.cf_list[j];
    const int f = e >= 0 ? e : ~e;
    const double A = m.f_area[f];
    const double out = (e >= 0 ? mdot[f] : -mdot[f]) * A;  // mass leaving the cell through f
    if (out > 0.) conv += out;
    const int o = e >= 0 ? m.f_neighbor[f] : m.f_parent[f];
    const double l0 = m.c_x[o] - m.c_x[c], l1 = m.c_x[nt + o] - m.c_x[nt + c], l2 = m.c_x[2 * nt + o] - m.c_x[2 * nt + c];
    const double il = A / sqrt(l0 * l0 + l1 * l1 + l2 * l2);
    dk0 += (mu + KOmega::sigma_k * mutf[f]) * il;
    dk1 += (mu + KOmega::sigma_omega * mutf[f]) * il;
  }
  const double t = rho * vol[c] / dt[c];
  dk[c] = t + conv + dk0 + KOmega::beta_star * rho * om * vol[c];
  dk[nc + c] = t + conv + dk1 + 2. * KOmega::beta * rho * om * vol[c];
}

// z = M^-1 v: flow rows through the inverse blocks, k and omega rows by the
// diagonal; v carries the equation weights wr (removed first).
__global__ void k_kw_prec(int nc, const double *__restrict__ Minv, const double *__restrict__ dk,
                          const KwIter *__restrict__ it, const double *__restrict__ v, double *__restrict__ z) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  const Wt7 &iwr = it->iwr;
  double b[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) b[k] = iwr.s[k] * v[k * nc + c];
#pragma unroll
  for (int i = 0; i < 5; ++i) {
    double s = 0.;
#pragma unroll
    for (int k = 0; k < 5; ++k) s += Minv[(5 * i + k) * nc + c] * b[k];
    z[i * nc + c] = s;
  }
  z[5 * nc + c] = iwr.s[5] * v[5 * nc + c] / dk[c];
  z[6 * nc + c] = iwr.s[6] * v[6 * nc + c] / dk[nc + c];
}

// part[j * gridDim.x + b] = block b's share of V_j . w (j < nv)
// The column's last block adds its partials (in block order, strided over
// the block's threads) and re-arms the column's counter.
__device__ void kw_last_block_sum(int nparts, const double *part, double *__restrict__ out, unsigned *__restrict__ count) {
  __shared__ unsigned ticket;
  __shared__ double shs[8];
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) ticket = atomicAdd(count, 1u);
  __syncthreads();
  if (ticket != (unsigned)nparts - 1u) return;
  __threadfence();
  double s = 0.;
  for (int i = threadIdx.x; i < nparts; i += blockDim.x) s += __ldcg(part + i);
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) shs[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += shs[k];
    *out = t;
    *count = 0u;
  }
}
// part[j][block] = this block's share of V_j . w; with out and count (one
// counter per column, 256-thread blocks) the column's last block also writes
// out[j], so the sums stay on the device
__global__ void k_kw_dots(int n, int nv, const double *__restrict__ V, size_t ld, const double *__restrict__ w,
                          double *__restrict__ part, double *__restrict__ out = nullptr,
                          unsigned *__restrict__ count = nullptr) {
  const int j = blockIdx.y;
  const double *a = V + (size_t)j * ld;
  double s = 0.;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) s += a[i] * w[i];
  __shared__ double sh[32];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    double t = threadIdx.x < blockDim.x / 32 ? sh[threadIdx.x] : 0.;
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (threadIdx.x == 0) part[(size_t)j * gridDim.x + blockIdx.x] = t;
  }
  if (count) kw_last_block_sum(gridDim.x, part + (size_t)j * gridDim.x, out + j, count + j);
}
// y = x / sqrt(*ss) where *ss > 0
__global__ void k_kw_scale_rsqrt(int n, const double *__restrict__ ss, const double *__restrict__ x, double *__restrict__ y) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const double q = *ss;
  if (i < n && q > 0.) y[i] = x[i] / sqrt(q);
}

// w -= sum_j h[j] V_j (h in device memory), then optionally out = w * scale
__global__ void k_kw_sub(int n, int nv, const double *__restrict__ V, size_t ld, const double *__restrict__ h,
                         double *__restrict__ w) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double s = w[i];
  for (int j = 0; j < nv; ++j) s -= h[j] * V[(size_t)j * ld + i];
  w[i] = s;
}
__global__ void k_kw_scale(int n, double a, const double *__restrict__ x, double *__restrict__ y) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] = a * x[i];
}
__global__ void k_kw_combo(int n, int nv, const double *__restrict__ V, size_t ld, const double *__restrict__ yk,
                           double *__restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double s = 0.;
  for (int j = 0; j < nv; ++j) s += yk[j] * V[(size_t)j * ld + i];
  out[i] = s;
}

// largest relative change |dp|/(p+Pref), |dT|/(T+Tref) and relative
// decrease -dk/k, -domega/omega (ordered-key maxima in key[0], key[1])
__global__ void k_kw_change(DevCase cs, int nc, const double *__restrict__ X, const double *__restrict__ dX,
                            unsigned long long *__restrict__ key) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nc) return;
  const double a = fmax(fabs(dX[c]) / fabs(X[c] + cs.Pref), fabs(dX[4 * nc + c]) / fabs(X[4 * nc + c] + cs.Tref));
  const double b = fmax(-dX[5 * nc + c] / X[5 * nc + c], -dX[6 * nc + c] / X[6 * nc + c]);
  atomicMax(&key[0], okey(a == a ? a : 1e300));
  atomicMax(&key[1], okey(b == b ? b : 1e300));
}

// X += alpha dX with k, omega kept at or above their lower limits
__global__ void k_kw_update(int nc, double *__restrict__ X, const double *__restrict__ dX, double alpha, double klow,
                            double omlow) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kNv * nc) return;
  double x = X[i] + alpha * dX[i];
  if (i >= 5 * nc && i < 6 * nc) x = fmax(x, klow);
  if (i >= 6 * nc) x = fmax(x, omlow);
  X[i] = x;
}

// Device buffers of one coupled Newton solve.
struct KwSolve {
  DBuf<double> X, Xsave, F0, F1, Jz, dt, vol, Minv, JL, JR, rowmag, dk, Vb, w, z, part, h, x, dX;
  DBuf<unsigned long long> key;
  std::vector<double> hpart;
  // device-side Gram-Schmidt: coefficients h1[mdim+1], h2[mdim+1], |w|^2,
  // |z|^2; one counter per dot-product column
  DBuf<double> hd;
  DBuf<unsigned> cnt;
  double *hh = nullptr;  // page-locked copy of hd
  DBuf<KwIter> it;
  // one captured Arnoldi step per basis index, for the J.v mode graph_mode
  std::vector<cudaGraphExec_t> graphs;
  int graph_mode = -1;
  void alloc_gs(int mdim, cudaStream_t s) {
    hd.alloc(2 * (size_t)(mdim + 1) + 2);
    cnt.alloc((size_t)mdim + 1);
    it.alloc(1);
    CK(cudaMemsetAsync(cnt.p, 0, sizeof(unsigned) * (mdim + 1), s));
    CK(cudaMallocHost((void **)&hh, sizeof(double) * hd.n));
  }
  ~KwSolve() {
    for (cudaGraphExec_t g : graphs)
      if (g) cudaGraphExecDestroy(g);
    if (hh) cudaFreeHost(hh);
  }
};

// sum of the per-block partials of nv dot products, in block order (host)
static void kw_dots(fcfd_ctx *x, KwSolve &S, int n, int nv, const double *V, size_t ld, const double *w, double *out) {
  cudaStream_t s = x->stream;
  k_kw_dots<<<dim3(kRedBlk, nv), 256, 0, s>>>(n, nv, V, ld, w, S.part.p);
  S.hpart.resize((size_t)kRedBlk * nv);
  CK(cudaMemcpyAsync(S.hpart.data(), S.part.p, sizeof(double) * kRedBlk * nv, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  for (int j = 0; j < nv; ++j) {
    double t = 0.;
    for (int b = 0; b < kRedBlk; ++b) t += S.hpart[(size_t)j * kRedBlk + b];
    out[j] = t;
  }
}

// F = F(X) into out (SoA [7][nc]); X + eps z when z is given.  Leaves the
// chain's state (gradients, limiters, mdot, eddy viscosities) of that point
// in x->p64 / x->rans->b.
static void kw_residual(fcfd_ctx *x, const double *X, const double *z, double eps, double *out) {
  const DevMesh &m = x->dm;
  cudaStream_t s = x->stream;
  const int gc = (m.nc + 255) / 256;
  RansBuf<double> &b = x->rans->b;
  k_x_load<<<gc, 256, 0, s>>>(m.nc, m.nt, X, z, eps, x->p64.W.p, b.K.p);
  rans_chain<double, false>(x, x->p64, b, x->mdot.p, x->wl.p, out, b.RK.p);
  k_rk_planes<<<gc, 256, 0, s>>>(m.nc, b.RK.p, out);
}

// Jz of the coupled FP32 tangent chain at X along z
static void kw_tangent32(fcfd_ctx *x, const double *X, const double *z, double *Jz) {
  const DevMesh &m = x->dm;
  cudaStream_t s = x->stream;
  const int gc = (m.nc + 255) / 256;
  if (!x->pjv32.ready) x->pjv32.alloc(m.nc, m.nf, m.nb);
  RansBuf<Dual<float>> &d = x->rans->f;
  if (!d.ready) d.alloc(m.nc, m.nt, m.nf);
  k_x_load_dual<<<gc, 256, 0, s>>>(m.nc, m.nt, X, z, x->pjv32.W.p, d.K.p);
  rans_chain<Dual<float>, false>(x, x->pjv32, d, d.mdot.p, d.wl.p, x->pjv32.R.p, d.RK.p);
  k_dual_planes<<<gc, 256, 0, s>>>(m.nc, x->pjv32.R.p, d.RK.p, Jz);
}

}  // namespace kwn
}  // namespace fcfd

using namespace fcfd::kwn;

// One linearised backward-Euler solve of the coupled system at S.X (its
// residual in S.F0, local time steps in S.dt): the flow rows' block inverses
// and the k-omega diagonal at X, then GMRES(mdim), one cycle, on
// wr (D/dt - J) M^-1 u = wr F0 stopped at |r| <= krtol |wr F0| or kabstol;
// dX = M^-1 u into S.dX.  mode 0: J.v by an FP64 finite difference of the
// coupled residual, else the FP32 coupled tangent.  Returns the Krylov
// iterations.  Shared by the coupled Newton solve and the time-marching
// driver of turbulent decks.
static int kw_linear_step(fcfd_ctx *x, KwSolve &S, int mdim, int mode, double krtol, double kabstol, const Wt7 &wr,
                          const Wt7 &iwr) {
  const DevMesh &m = x->dm;
  const int nc = m.nc, n = kNv * nc;
  cudaStream_t s = x->stream;
  const int gc = (nc + 255) / 256, gn = (n + 255) / 256;
  auto norms = [&](const double *F, double out[kNv]) {
    for (int v = 0; v < kNv; ++v) {
      double d;
      kw_dots(x, S, nc, 1, F + (size_t)v * nc, 0, F + (size_t)v * nc, &d);
      out[v] = std::sqrt(d);
    }
  };
  ns_block_inverse(x, S.X.p, S.vol.p, S.dt.p, x->rans->b.mutf.p, S.JL.p, S.JR.p, S.Minv.p, S.rowmag.p);
  k_kw_diag<<<gc, 256, 0, s>>>(x->cs, m, S.X.p, S.vol.p, S.dt.p, x->mdot.p, x->rans->b.mutf.p, S.dk.p);
  // GMRES(m), one cycle, on wr (D - J) M^-1 u = wr F0, dX = M^-1 u
  // |S^-1 X| for the finite-difference step (S: the equations' scales)
  double xn = 0.;
  {
    double d[kNv];
    norms(S.X.p, d);
    const double ref[kNv] = {std::fabs(x->cs.Pref) + d[0] / std::sqrt((double)nc), 0., 0., 0.,
                             std::fabs(x->cs.Tref) + d[4] / std::sqrt((double)nc), d[5] / std::sqrt((double)nc),
                             d[6] / std::sqrt((double)nc)};
    double U = std::sqrt(d[1] * d[1] + d[2] * d[2] + d[3] * d[3]) / std::sqrt((double)nc);
    for (int v = 0; v < kNv; ++v) {
      const double r = (v >= 1 && v <= 3) ? U : ref[v];
      if (r > 0.) xn += (d[v] / r) * (d[v] / r);
    }
    xn = std::sqrt(xn);
  }
  for (int v = 0; v < kNv; ++v)
    k_kw_scale<<<gc, 256, 0, s>>>(nc, wr.s[v], S.F0.p + (size_t)v * nc, S.w.p + (size_t)v * nc);
  double beta;
  kw_dots(x, S, n, 1, S.w.p, 0, S.w.p, &beta);
  beta = std::sqrt(beta);
  int kit = 0;
  std::vector<double> H((size_t)(mdim + 1) * mdim, 0.), g(mdim + 1, 0.), cs_(mdim), sn(mdim);
  g[0] = beta;
  if (beta > 0.) {
    k_kw_scale<<<gn, 256, 0, s>>>(n, 1. / beta, S.w.p, S.Vb.p);
    // per linear step constants on the device (the captured steps read them)
    KwIter hit;
    hit.wr = wr;
    hit.iwr = iwr;
    hit.eps_num = 1.4901161193847656e-08 * (1. + xn);
    CK(cudaMemcpyAsync(S.it.p, &hit, sizeof(KwIter), cudaMemcpyHostToDevice, s));
    if (mode != 0) {
      // tangent buffers before any capture
      if (!x->pjv32.ready) x->pjv32.alloc(m.nc, m.nf, m.nb);
      if (!x->rans->f.ready) x->rans->f.alloc(m.nc, m.nt, m.nf);
    }
    if (S.graph_mode != mode) {
      for (cudaGraphExec_t &g : S.graphs)
        if (g) { CK(cudaGraphExecDestroy(g)); g = nullptr; }
      S.graphs.assign(mdim, nullptr);
      S.graph_mode = mode;
    }
    // the Gram-Schmidt coefficients, |w|^2 and |z|^2 stay on the device
    // (fused dot products); one Arnoldi step is one captured graph, replayed
    // with one copy back and one synchronisation
    double *h1 = S.hd.p, *h2 = S.hd.p + (mdim + 1), *hw = S.hd.p + 2 * (mdim + 1), *zz = hw + 1;
    for (int j = 0; j < mdim; ++j) {
      if (!S.graphs[j]) {
        double *vj = S.Vb.p + (size_t)j * n;
        cudaGraph_t gr = nullptr;
        CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        // z = M^-1 v_j, then w = wr (D z - J z)
        k_kw_prec<<<gc, 256, 0, s>>>(nc, S.Minv.p, S.dk.p, S.it.p, vj, S.z.p);
        if (mode == 0) {
          // eps = sqrt(eps_mach) (1 + |S^-1 X|) / |z|, |z| read on the device
          k_kw_dots<<<dim3(kRedBlk, 1), 256, 0, s>>>(n, 1, S.z.p, 0, S.z.p, S.part.p, zz, S.cnt.p);
          k_x_load<<<gc, 256, 0, s>>>(m.nc, m.nt, S.X.p, S.z.p, 0., x->p64.W.p, x->rans->b.K.p, S.it.p, zz);
          rans_chain<double, false>(x, x->p64, x->rans->b, x->mdot.p, x->wl.p, S.F1.p, x->rans->b.RK.p);
          k_rk_planes<<<gc, 256, 0, s>>>(m.nc, x->rans->b.RK.p, S.F1.p);
          k_kw_matvec<<<gc, 256, 0, s>>>(x->cs, nc, S.X.p, S.vol.p, S.dt.p, S.z.p, S.F1.p, S.F0.p, 0., S.it.p, S.w.p, zz);
        } else {
          kw_tangent32(x, S.X.p, S.z.p, S.Jz.p);
          k_kw_matvec<<<gc, 256, 0, s>>>(x->cs, nc, S.X.p, S.vol.p, S.dt.p, S.z.p, S.Jz.p, nullptr, 0., S.it.p, S.w.p);
        }
        // classical Gram-Schmidt, twice
        k_kw_dots<<<dim3(kRedBlk, j + 1), 256, 0, s>>>(n, j + 1, S.Vb.p, (size_t)n, S.w.p, S.part.p, h1, S.cnt.p);
        k_kw_sub<<<gn, 256, 0, s>>>(n, j + 1, S.Vb.p, (size_t)n, h1, S.w.p);
        k_kw_dots<<<dim3(kRedBlk, j + 1), 256, 0, s>>>(n, j + 1, S.Vb.p, (size_t)n, S.w.p, S.part.p, h2, S.cnt.p);
        k_kw_sub<<<gn, 256, 0, s>>>(n, j + 1, S.Vb.p, (size_t)n, h2, S.w.p);
        k_kw_dots<<<dim3(kRedBlk, 1), 256, 0, s>>>(n, 1, S.w.p, 0, S.w.p, S.part.p, hw, S.cnt.p);
        k_kw_scale_rsqrt<<<gn, 256, 0, s>>>(n, hw, S.w.p, S.Vb.p + (size_t)(j + 1) * n);
        CK(cudaMemcpyAsync(S.hh, S.hd.p, sizeof(double) * S.hd.n, cudaMemcpyDeviceToHost, s));
        CK(cudaStreamEndCapture(s, &gr));
        CK(cudaGraphInstantiate(&S.graphs[j], gr, 0));
        CK(cudaGraphDestroy(gr));
      }
      CK(cudaGraphLaunch(S.graphs[j], s));
      CK(cudaStreamSynchronize(s));
      const double hn = std::sqrt(S.hh[2 * (mdim + 1)]);
      for (int i = 0; i <= j; ++i) H[(size_t)i * mdim + j] = S.hh[i] + S.hh[mdim + 1 + i];
      H[(size_t)(j + 1) * mdim + j] = hn;
      // Givens rotations of the new column
      for (int i = 0; i < j; ++i) {
        const double a = H[(size_t)i * mdim + j], b = H[(size_t)(i + 1) * mdim + j];
        H[(size_t)i * mdim + j] = cs_[i] * a + sn[i] * b;
        H[(size_t)(i + 1) * mdim + j] = -sn[i] * a + cs_[i] * b;
      }
      const double a = H[(size_t)j * mdim + j], b = H[(size_t)(j + 1) * mdim + j];
      const double r = std::hypot(a, b);
      cs_[j] = r > 0. ? a / r : 1.;
      sn[j] = r > 0. ? b / r : 0.;
      H[(size_t)j * mdim + j] = r;
      H[(size_t)(j + 1) * mdim + j] = 0.;
      g[j + 1] = -sn[j] * g[j];
      g[j] = cs_[j] * g[j];
      kit = j + 1;
      if (std::fabs(g[j + 1]) <= krtol * beta || std::fabs(g[j + 1]) <= kabstol || hn == 0.) break;
    }
    // y = H^-1 g, u = V y, dX = M^-1 u
    std::vector<double> y(kit, 0.);
    for (int i = kit - 1; i >= 0; --i) {
      double t = g[i];
      for (int k = i + 1; k < kit; ++k) t -= H[(size_t)i * mdim + k] * y[k];
      y[i] = t / H[(size_t)i * mdim + i];
    }
    CK(cudaMemcpyAsync(S.h.p, y.data(), sizeof(double) * kit, cudaMemcpyHostToDevice, s));
    k_kw_combo<<<gn, 256, 0, s>>>(n, kit, S.Vb.p, (size_t)n, S.h.p, S.x.p);
    k_kw_prec<<<gc, 256, 0, s>>>(nc, S.Minv.p, S.dk.p, S.it.p, S.x.p, S.dX.p);
  } else if (!std::isfinite(beta)) {
    // a non-finite right-hand side: a NaN update, which the update's NaN
    // check reports as divergence (as the reference's NaN check would)
    k_kw_scale<<<gn, 256, 0, s>>>(n, std::numeric_limits<double>::quiet_NaN(), S.w.p, S.dX.p);
  } else {
    CK(cudaMemsetAsync(S.dX.p, 0, sizeof(double) * n, s));
  }
  return kit;
}

namespace fcfd {

// ---- the implicit step of the time-marching driver for turbulent decks
// (fcfd_run): one coupled backward-Euler solve per time step on
// X = (p,u,v,w,T,k,omega), where the reference solves the flow system and
// then the k-omega system (ns.cc:104-118, rans.cc:85-98) -- the same steady
// state, one linear solve instead of two.
struct KwDriver {
  KwSolve S;
  Wt7 wr, iwr;
  int mdim = 10;
};

// X += dX with the reference's k-omega update limits (rans.cc:214-220: k
// kept in [klow, khigh], omega above omegalow), NaN/Inf updates flagged (err
// bit 8), and per block the sums of dp^2, |dV|^2, dT^2, dk^2, domega^2 over
// dt^2 (update_variables of both solvers, ns.cc:338-396, rans.cc:193-255)
__global__ void k_kw_drive_update(int nc, double *__restrict__ X, const double *__restrict__ dX,
                                  const double *__restrict__ dt, double klow, double khigh, double omlow,
                                  double *__restrict__ part, int *__restrict__ err) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  double r[5] = {0., 0., 0., 0., 0.};
  if (c < nc) {
    double d[kNv];
    bool bad = false;
    for (int k = 0; k < kNv; ++k) {
      d[k] = dX[(size_t)k * nc + c];
      if (!isfinite(d[k])) bad = true;
    }
    if (bad) atomicOr(err, 8);
    const double kk = X[(size_t)5 * nc + c], om = X[(size_t)6 * nc + c];
    d[5] = fmax(-1. * (kk - klow), d[5]);
    d[5] = fmin(khigh - kk, d[5]);
    d[6] = fmax(-1. * (om - omlow), d[6]);
    for (int k = 0; k < kNv; ++k) X[(size_t)k * nc + c] += d[k];
    const double dt2 = dt[c] * dt[c];
    r[0] = d[0] * d[0] / dt2;
    r[1] = d[1] * d[1] / dt2 + d[2] * d[2] / dt2 + d[3] * d[3] / dt2;
    r[2] = d[4] * d[4] / dt2;
    r[3] = d[5] * d[5] / dt2;
    r[4] = d[6] * d[6] / dt2;
  }
  __shared__ double sh[5][8];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int i = 0; i < 5; ++i) {
    double t = r[i];
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (lane == 0) sh[i][wid] = t;
  }
  __syncthreads();
  if (threadIdx.x < 5) {
    double t = 0.;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += sh[threadIdx.x][k];
    part[(size_t)blockIdx.x * 5 + threadIdx.x] = t;
  }
}

void *kw_driver_create(fcfd_ctx *x, const double *W, const double *K, int mdim) {
  if (!x->rans) throw Error(FCFD_ERR_INPUT, "the case has no turbulence model");
  const DevMesh &m = x->dm;
  const int nc = m.nc, n = kNv * nc;
  cudaStream_t s = x->stream;
  std::unique_ptr<KwDriver> d(new KwDriver());
  d->mdim = mdim > 0 ? mdim : 10;
  KwSolve &S = d->S;
  S.X.alloc(n); S.Xsave.alloc(n); S.F0.alloc(n); S.F1.alloc(n); S.Jz.alloc(n); S.dt.alloc(nc); S.vol.alloc(nc);
  S.Minv.alloc(25 * (size_t)nc); S.JL.alloc(25 * (size_t)m.nf); S.JR.alloc(25 * (size_t)m.nf);
  S.rowmag.alloc(5 * (size_t)nc); S.dk.alloc(2 * (size_t)nc);
  S.Vb.alloc((size_t)(d->mdim + 1) * n); S.w.alloc(n); S.z.alloc(n); S.part.alloc((size_t)kRedBlk * (d->mdim + 1));
  S.h.alloc(d->mdim + 1); S.x.alloc(n); S.dX.alloc(n); S.key.alloc(2);
  S.alloc_gs(d->mdim, s);
  std::vector<double> hx((size_t)n);
  for (int c = 0; c < nc; ++c) {
    for (int v = 0; v < 5; ++v) hx[(size_t)v * nc + c] = W[5 * (size_t)c + v];
    for (int v = 0; v < 2; ++v) hx[(size_t)(5 + v) * nc + c] = K[2 * (size_t)c + v];
  }
  CK(cudaMemcpyAsync(S.X.p, hx.data(), sizeof(double) * n, cudaMemcpyHostToDevice, s));
  std::vector<double> vol(x->mesh->c_volume.begin(), x->mesh->c_volume.begin() + nc);
  CK(cudaMemcpyAsync(S.vol.p, vol.data(), sizeof(double) * nc, cudaMemcpyHostToDevice, s));
  CK(cudaStreamSynchronize(s));
  return d.release();
}

void kw_driver_destroy(void *p) { delete static_cast<KwDriver *>(p); }

// F0 = the coupled residual at X; it also loads X's flow state into the
// residual pipeline (x->p64: the time step and loads read it).  The Krylov
// equation weights are the inverse norms of this residual (momentum as
// one), formed anew at every step so that a run continued from restart files
// takes the same steps as an uninterrupted one.
void kw_driver_residual(fcfd_ctx *x, void *p) {
  KwDriver &d = *static_cast<KwDriver *>(p);
  KwSolve &S = d.S;
  const int nc = x->dm.nc;
  kw_residual(x, S.X.p, nullptr, 0., S.F0.p);
  check_err(x);
  {
    double r0[kNv];
    for (int v = 0; v < kNv; ++v) {
      double q;
      kw_dots(x, S, nc, 1, S.F0.p + (size_t)v * nc, 0, S.F0.p + (size_t)v * nc, &q);
      r0[v] = std::sqrt(q);
    }
    const double m0 = std::sqrt(r0[1] * r0[1] + r0[2] * r0[2] + r0[3] * r0[3]);
    for (int v = 0; v < kNv; ++v) {
      const double r = (v >= 1 && v <= 3) ? m0 : r0[v];
      d.wr.s[v] = r > 0. ? 1. / r : 1.;
      d.iwr.s[v] = 1. / d.wr.s[v];
    }
  }
}

// the implicit solve at X with local time steps dt (device, [nc]); dX in the driver state
int kw_driver_step(fcfd_ctx *x, void *p, const double *dt, int mode, double krtol, double kabstol) {
  KwDriver &d = *static_cast<KwDriver *>(p);
  CK(cudaMemcpyAsync(d.S.dt.p, dt, sizeof(double) * x->dm.nc, cudaMemcpyDeviceToDevice, x->stream));
  return kw_linear_step(x, d.S, d.mdim, mode, krtol, kabstol, d.wr, d.iwr);
}

// X += dX (limits as k_kw_drive_update); part: 5 partial sums per 256-cell block
void kw_driver_update(fcfd_ctx *x, void *p, const double *dt, double *part, int *err) {
  KwDriver &d = *static_cast<KwDriver *>(p);
  const fcfd_case &cs = *x->case_ptr;
  const int nc = x->dm.nc;
  k_kw_drive_update<<<(nc + 255) / 256, 256, 0, x->stream>>>(nc, d.S.X.p, d.S.dX.p, dt, cs.k_low, cs.k_high, cs.omega_low,
                                                               part, err);
  CK(cudaGetLastError());
}

// host copies of the state: W[nc][5], K[nc][2] and (mut, may be null) the
// cells' eddy viscosity of the last residual evaluation
void kw_driver_state(fcfd_ctx *x, void *p, double *W, double *K, double *mut) {
  KwDriver &d = *static_cast<KwDriver *>(p);
  const int nc = x->dm.nc, n = kNv * nc;
  std::vector<double> hx((size_t)n);
  CK(cudaMemcpyAsync(hx.data(), d.S.X.p, sizeof(double) * n, cudaMemcpyDeviceToHost, x->stream));
  if (mut) CK(cudaMemcpyAsync(mut, x->rans->b.mut.p, sizeof(double) * nc, cudaMemcpyDeviceToHost, x->stream));
  CK(cudaStreamSynchronize(x->stream));
  for (int c = 0; c < nc; ++c) {
    for (int v = 0; v < 5; ++v) W[5 * (size_t)c + v] = hx[(size_t)v * nc + c];
    for (int v = 0; v < 2; ++v) K[2 * (size_t)c + v] = hx[(size_t)(5 + v) * nc + c];
  }
}

}  // namespace fcfd

extern "C" int fcfd_rans_newton_solve(fcfd_ctx *x, double *W, double *K, const fcfd_newton_opts *o,
                                      fcfd_newton_report *rep) {
  try {
    if (!x || !W || !K || !o || !rep) throw Error(FCFD_ERR_INPUT, "null argument");
    if (!x->rans) throw Error(FCFD_ERR_INPUT, "the case has no turbulence model");
    CK(cudaSetDevice(x->device));
    const DevMesh &m = x->dm;
    const int nc = m.nc, n = kNv * nc;
    cudaStream_t s = x->stream;
    const int gc = (nc + 255) / 256, gn = (n + 255) / 256;
    std::memset(rep, 0, sizeof(*rep));
    rep->seconds_to_tol = -1.;
    const int mdim = o->krylov_dim > 0 ? o->krylov_dim : 30;
    const int mode = o->jvp_mode;  // 0: FD in FP64, else the FP32 tangent chain
    KwSolve S;
    S.X.alloc(n); S.Xsave.alloc(n); S.F0.alloc(n); S.F1.alloc(n); S.Jz.alloc(n); S.dt.alloc(nc); S.vol.alloc(nc);
    S.Minv.alloc(25 * (size_t)nc); S.JL.alloc(25 * (size_t)m.nf); S.JR.alloc(25 * (size_t)m.nf);
    S.rowmag.alloc(5 * (size_t)nc); S.dk.alloc(2 * (size_t)nc);
    S.Vb.alloc((size_t)(mdim + 1) * n); S.w.alloc(n); S.z.alloc(n); S.part.alloc((size_t)kRedBlk * (mdim + 1));
    S.h.alloc(mdim + 1); S.x.alloc(n); S.dX.alloc(n); S.key.alloc(2);
    S.alloc_gs(mdim, s);
    // X from the host's AoS W[nc][5], K[nc][2]
    {
      std::vector<double> hx((size_t)n);
      for (int c = 0; c < nc; ++c) {
        for (int v = 0; v < 5; ++v) hx[(size_t)v * nc + c] = W[5 * (size_t)c + v];
        for (int v = 0; v < 2; ++v) hx[(size_t)(5 + v) * nc + c] = K[2 * (size_t)c + v];
      }
      CK(cudaMemcpyAsync(S.X.p, hx.data(), sizeof(double) * n, cudaMemcpyHostToDevice, s));
      std::vector<double> vol(x->mesh->c_volume.begin(), x->mesh->c_volume.begin() + nc);
      CK(cudaMemcpyAsync(S.vol.p, vol.data(), sizeof(double) * nc, cudaMemcpyHostToDevice, s));
      CK(cudaStreamSynchronize(s));
    }
    const double klow = x->case_ptr->k_low, omlow = x->case_ptr->omega_low;
    auto t0 = std::chrono::steady_clock::now();
    auto seconds = [&]() { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); };
    // per-equation residual norms (momentum x, y, z together)
    double r0[kNv], rn[kNv];
    auto norms = [&](const double *F, double out[kNv]) {
      const int nd = 1;
      for (int v = 0; v < kNv; ++v) {
        double d;
        kw_dots(x, S, nc, nd, F + (size_t)v * nc, 0, F + (size_t)v * nc, &d);
        out[v] = std::sqrt(d);
      }
    };
    kw_residual(x, S.X.p, nullptr, 0., S.F0.p);
    check_err(x);
    norms(S.F0.p, r0);
    auto mom = [](const double r[kNv]) { return std::sqrt(r[1] * r[1] + r[2] * r[2] + r[3] * r[3]); };
    const double m0 = mom(r0);
    std::copy(r0, r0 + kNv, rn);
    // equation weights: the inverse of each equation's initial norm (momentum as one)
    Wt7 wr, iwr;
    for (int v = 0; v < kNv; ++v) {
      const double r = (v >= 1 && v <= 3) ? m0 : r0[v];
      wr.s[v] = r > 0. ? 1. / r : 1.;
      iwr.s[v] = 1. / wr.s[v];
    }
    rep->res0 = r0[0];
    const double cfl0 = o->cfl0 > 0 ? o->cfl0 : 1.;
    const double cflmax = o->cfl_max > 0 ? o->cfl_max : 1e6;
    double cfl = cfl0, cfl_prev = cfl0;
    const int maxit = o->max_newton > 0 ? o->max_newton : 200;
    const int hist = (int)(sizeof(rep->history) / sizeof(rep->history[0]));
    const double krtol = o->krylov_rtol > 0 ? o->krylov_rtol : 1e-2;
    int status = FCFD_ERR_NOT_CONVERGED, rejects = 0;
    // combined drop of all equations (the largest per-equation drop)
    auto drop_all = [&](const double r[kNv]) {
      double d = 0.;
      for (int v = 0; v < kNv; ++v) {
        if (v >= 1 && v <= 3) continue;
        if (r0[v] > 0.) d = std::max(d, r[v] / r0[v]);
      }
      if (m0 > 0.) d = std::max(d, mom(r) / m0);
      return d;
    };
    for (int it = 0; it < maxit; ++it) {
      const double rm = rn[0] / r0[0], ra = drop_all(rn);
      if (it < hist) { rep->history[it] = rm; rep->seconds_history[it] = seconds(); }
      if (rm <= o->tol && rep->seconds_to_tol < 0.) rep->seconds_to_tol = seconds();
      if ((o->stop_all_rows ? ra : rm) <= o->tol) { status = FCFD_OK; break; }
      if (o->max_seconds > 0 && seconds() > o->max_seconds) break;
      // time step, preconditioner at X (the chain's state of F0 is current)
      k_local_dt<double><<<gc, 256, 0, s>>>(x->cs, m, x->p64.W.p, S.dt.p, cfl, nullptr);
      CK(cudaMemcpyAsync(S.Xsave.p, S.X.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
      const int kit = kw_linear_step(x, S, mdim, mode, krtol, 0., wr, iwr);
      rep->krylov_iterations += kit;
      // relaxation: |dp/p|, |dT/T| <= 0.2
      CK(cudaMemsetAsync(S.key.p, 0, 2 * sizeof(unsigned long long), s));
      k_kw_change<<<gc, 256, 0, s>>>(x->cs, nc, S.X.p, S.dX.p, S.key.p);
      unsigned long long kh[2];
      CK(cudaMemcpyAsync(kh, S.key.p, sizeof(kh), cudaMemcpyDeviceToHost, s));
      CK(cudaStreamSynchronize(s));
      auto unkey = [](unsigned long long k) {
        unsigned long long b = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
        double d;
        std::memcpy(&d, &b, sizeof(d));
        return d;
      };
      // p and T limit the step; k and omega are clipped at their lower limits
      // instead (one cell's k heading for zero would otherwise stall the step)
      const double da = unkey(kh[0]);
      double alpha = 1.;
      if (da > 0.2) alpha = std::min(alpha, 0.2 / da);
      k_kw_update<<<gn, 256, 0, s>>>(nc, S.X.p, S.dX.p, alpha, klow, omlow);
      kw_residual(x, S.X.p, nullptr, 0., S.F1.p);
      int herr = 0;
      CK(cudaMemcpyAsync(&herr, x->err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
      CK(cudaStreamSynchronize(s));
      if (herr) CK(cudaMemsetAsync(x->err.p, 0, sizeof(int), s));
      double rnew[kNv];
      norms(S.F1.p, rnew);
      rep->newton_iterations = it + 1;
      bool finite = !herr;
      for (int v = 0; v < kNv; ++v) finite = finite && std::isfinite(rnew[v]);
      if (!finite) {
        if (++rejects > 12) { status = FCFD_ERR_DIVERGED; break; }
        CK(cudaMemcpyAsync(S.X.p, S.Xsave.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
        kw_residual(x, S.X.p, nullptr, 0., S.F0.p);
        cfl = std::max(cfl * 0.25, 1e-3);
        cfl_prev = cfl;
        continue;
      }
      rejects = 0;
      CK(cudaMemcpyAsync(S.F0.p, S.F1.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
      std::copy(rnew, rnew + kNv, rn);
      rep->last_cfl = cfl;
      // switched evolution/relaxation on the mass residual (cfl_mode 1) or on
      // the largest per-equation drop (cfl_mode 2)
      const double dr = o->cfl_mode == 2 ? drop_all(rn) : rn[0] / r0[0];
      double next = cfl0 * std::pow(1. / std::max(dr, 1e-300), o->ser_exponent > 0 ? o->ser_exponent : 1.);
      next = std::min(next, cfl_prev * 2.);
      cfl_prev = cfl;
      cfl = std::min(std::max(next, 1e-3), cflmax);
    }
    CK(cudaStreamSynchronize(s));
    rep->wall_seconds = seconds();
    rep->res_final = rn[0];
    rep->rows_final[0] = rn[0] / r0[0];
    rep->rows_final[1] = m0 > 0. ? mom(rn) / m0 : 0.;
    rep->rows_final[2] = r0[4] > 0. ? rn[4] / r0[4] : 0.;
    rep->kw_final[0] = r0[5] > 0. ? rn[5] / r0[5] : 0.;
    rep->kw_final[1] = r0[6] > 0. ? rn[6] / r0[6] : 0.;
    rep->status = status;
    {
      std::vector<double> hx((size_t)n);
      CK(cudaMemcpy(hx.data(), S.X.p, sizeof(double) * n, cudaMemcpyDeviceToHost));
      for (int c = 0; c < nc; ++c) {
        for (int v = 0; v < 5; ++v) W[5 * (size_t)c + v] = hx[(size_t)v * nc + c];
        for (int v = 0; v < 2; ++v) K[2 * (size_t)c + v] = hx[(size_t)(5 + v) * nc + c];
      }
    }
    if (status != FCFD_OK) {
      set_last_error(status == FCFD_ERR_DIVERGED ? "k-omega Newton iteration diverged (NaN/Inf)"
                                                 : "k-omega Newton iteration did not reach the tolerance");
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
