// C ABI, device context and residual pipeline of libfcfd_b200.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <type_traits>
#include <vector>

#include "ctx.hpp"

namespace fcfd {

// defined in ghost.cu (compiled with -fmad=false)
extern template __global__ void k_ghost_minmax<double>(DevCase, DevMesh, double *, unsigned long long *, int *);
extern template __global__ void k_ghost_minmax<Dual<double>>(DevCase, DevMesh, Dual<double> *, unsigned long long *, int *);
extern template __global__ void k_ghost_minmax<Dual<float>>(DevCase, DevMesh, Dual<float> *, unsigned long long *, int *);

fcfd_case *read_deck(const std::string &path);
fcfd_mesh *build_mesh(const fcfd_raw_mesh &raw, fcfd_case &cs, const FaceInput *faces = nullptr);
void rcm_order(const fcfd_mesh &m, std::vector<int32_t> &perm);

static thread_local std::string g_last_error;
void set_last_error(const std::string &m) { g_last_error = m; }

template <class S>
void launch_chain(fcfd_ctx *x, Pipe<S> &P, S *Rout, bool aos_out, S *mo, S *wo, bool frozen_limiter) {
  const DevMesh &m = x->dm;
  DevCase csl = x->cs;
  csl.frozen_limiter = frozen_limiter ? 1 : 0;
  cudaStream_t s = x->stream;
  const int tb = 256;
  // the extrema and argx slots arrive armed (context set-up, then the
  // previous chain's gather)
  const bool need_ext = x->cs.limiter == 1 && x->cs.order != 1;
  const int ng = (m.nb + tb - 1) / tb + (need_ext ? kExtremaBlocks : 0);
  if (ng > 0)
    launch_k(x->pdl, k_ghost_minmax<S>, ng, tb, 0, s, x->cs, m, P.W.p, need_ext ? x->ext.p : nullptr, x->err.p);
  const int *argx = nullptr;
  if (!std::is_same<S, double>::value && x->cs.limiter == 1 && x->cs.order != 1) {
    k_argext<S><<<(m.nc + tb - 1) / tb, tb, 0, s>>>(m, P.W.p, x->ext.p, x->argx.p);
    argx = x->argx.p;
  }
  launch_grad_limiter<S>(csl, m, P.W.p, x->ext.p, argx, P.G.p, P.Lm.p, s, x->pdl);
  launch_faces<S>(x, P, (const S *)nullptr, mo, wo, s);
  const int gg = (5 * m.nc + tb - 1) / tb;
  if (aos_out)
    k_gather<S, true><<<gg, tb, 0, s>>>(m, P.D.p, Rout, x->ext.p, x->argx.p);
  else
    k_gather<S, false><<<gg, tb, 0, s>>>(m, P.D.p, Rout, x->ext.p, x->argx.p);
  CK(cudaGetLastError());
}

// Mixed-precision residual chain on x->p64 (state already in P.W): FP64
// ghosts, extrema, gradients and limiters; the stale-density outlet faces in
// FP64 on the side stream; the FP32 face pass with the shock-flagged faces
// in FP64 (mixed.cu); the FP64 gather into Rout ([nc][5]).
static void launch_mixed(fcfd_ctx *x, double shock_ratio, double *Rout) {
  const DevMesh &m = x->dm;
  cudaStream_t s = x->stream;
  Pipe<double> &P = x->p64;
  if (x->mx_count.n == 0) {
    x->mx_list.alloc(m.nf > 0 ? m.nf : 1);
    x->mx_count.alloc(1);
  }
  const int tb = 256;
  const bool need_ext = x->cs.limiter == 1 && x->cs.order != 1;
  const int ng = (m.nb + tb - 1) / tb + (need_ext ? kExtremaBlocks : 0);
  if (ng > 0) k_ghost_minmax<double><<<ng, tb, 0, s>>>(x->cs, m, P.W.p, need_ext ? x->ext.p : nullptr, x->err.p);
  launch_grad_limiter<double>(x->cs, m, P.W.p, x->ext.p, nullptr, P.G.p, P.Lm.p, s);
  CK(cudaMemsetAsync(x->mx_count.p, 0, sizeof(int), s));
  const bool side = m.n_outlet > 0;
  if (side) {
    CK(cudaEventRecord(x->ev_fork, s));
    CK(cudaStreamWaitEvent(x->side, x->ev_fork, 0));
    const int g = (m.n_outlet + 127) / 128;
    if (x->viscous)
      FCFD_BY_FLUX(x->cs.flux, k_face_flux<double, true, FX, true><<<g, 128, 0, x->side>>>(x->cs, m, P.W.p, P.G.p, P.Lm.p, P.stale.p, nullptr, P.D.p, nullptr, nullptr, x->err.p));
    else
      FCFD_BY_FLUX(x->cs.flux, k_face_flux<double, false, FX, true><<<g, 128, 0, x->side>>>(x->cs, m, P.W.p, P.G.p, P.Lm.p, P.stale.p, nullptr, P.D.p, nullptr, nullptr, x->err.p));
    CK(cudaEventRecord(x->ev_join, x->side));
  }
  launch_mixed_faces(x, shock_ratio, x->mx_list.p, x->mx_count.p, s);
  if (side) CK(cudaStreamWaitEvent(s, x->ev_join, 0));
  k_gather<double, true><<<(5 * m.nc + tb - 1) / tb, tb, 0, s>>>(m, P.D.p, Rout, x->ext.p, x->argx.p);
  CK(cudaGetLastError());
}

int check_err(fcfd_ctx *x) {
  int h = 0;
  CK(cudaMemcpyAsync(&h, x->err.p, sizeof(int), cudaMemcpyDeviceToHost, x->stream));
  CK(cudaStreamSynchronize(x->stream));
  if (h) {
    CK(cudaMemsetAsync(x->err.p, 0, sizeof(int), x->stream));
    if (h & ERR_SUPERSONIC_INLET) throw Error(FCFD_ERR_BC, "an inlet became supersonic; the thermodynamic state must be specified");
    throw Error(FCFD_ERR_BC, "invalid boundary condition specification");
  }
  return 0;
}

template void launch_chain<double>(fcfd_ctx *, Pipe<double> &, double *, bool, double *, double *, bool);
template void launch_chain<Dual<double>>(fcfd_ctx *, Pipe<Dual<double>> &, Dual<double> *, bool, Dual<double> *, Dual<double> *, bool);
template void launch_chain<Dual<float>>(fcfd_ctx *, Pipe<Dual<float>> &, Dual<float> *, bool, Dual<float> *, Dual<float> *, bool);

}  // namespace fcfd

using namespace fcfd;

#define API_BEGIN try {
#define API_END                                  \
  }                                              \
  catch (const fcfd::Error &e) {                 \
    fcfd::set_last_error(e.what());              \
    return e.code;                               \
  }                                              \
  catch (const std::exception &e) {              \
    fcfd::set_last_error(e.what());              \
    return FCFD_ERR_INPUT;                       \
  }                                              \
  return FCFD_OK;

extern "C" {

const char *fcfd_last_error(void) { return g_last_error.c_str(); }
const char *fcfd_version(void) { return "fcfd_b200 0.1 (sm_100a)"; }

int fcfd_case_from_deck(const char *deck_path, fcfd_case **out) {
  API_BEGIN
  if (!deck_path || !out) throw Error(FCFD_ERR_INPUT, "null argument");
  *out = read_deck(deck_path);
  API_END
}

void fcfd_case_destroy(fcfd_case *cs) { delete cs; }

int fcfd_case_summary(const fcfd_case *cs, double *dv, int32_t *iv, int32_t iv_len) {
  API_BEGIN
  const Material &m = cs->mat;
  double d[13] = {m.gamma, m.R, m.Pref, m.Tref, cs->Minf, cs->limiter_threshold, m.mu, m.lambda,
                  m.sut_mu_ref, m.sut_T_ref, m.sut_S, m.Pr, 0.};
  std::memcpy(dv, d, sizeof(d));
  int need = 7 + 4 * (int)cs->bc.size();
  if (iv_len < need) throw Error(FCFD_ERR_INPUT, "iv too small");
  iv[0] = cs->flux; iv[1] = cs->limiter; iv[2] = cs->order; iv[3] = m.sutherland; iv[4] = m.prandtl;
  iv[5] = (int)cs->bc.size(); iv[6] = cs->dimension;
  for (size_t b = 0; b < cs->bc.size(); ++b) {
    iv[7 + 4 * b] = cs->bc[b].type; iv[8 + 4 * b] = cs->bc[b].kind;
    iv[9 + 4 * b] = cs->bc[b].specified; iv[10 + 4 * b] = cs->bc[b].thermal;
  }
  API_END
}

int fcfd_mesh_create(const fcfd_raw_mesh *raw, const fcfd_case *cs, fcfd_mesh **out) {
  API_BEGIN
  if (!raw || !cs || !out) throw Error(FCFD_ERR_INPUT, "null argument");
  fcfd_case copy = *cs;
  *out = build_mesh(*raw, copy);
  API_END
}

void fcfd_mesh_destroy(fcfd_mesh *m) { delete m; }

int fcfd_mesh_sizes(const fcfd_mesh *m, int64_t *out) {
  API_BEGIN
  out[0] = m->nc; out[1] = m->nf; out[2] = m->nb; out[3] = m->nc + m->nb; out[4] = m->nnode;
  out[5] = (int64_t)m->st_keys.size(); out[6] = (int64_t)m->cf_list.size(); out[7] = (int64_t)m->nbr_list.size();
  API_END
}

int fcfd_mesh_connectivity(const fcfd_mesh *m, int32_t *face_parent, int32_t *face_neighbor, int32_t *face_bc,
                           int32_t *face_nodes, int32_t *cell_face_index, int32_t *cell_faces, int32_t *nbr_index,
                           int32_t *nbrs, int32_t *grad_index, int32_t *grad_keys) {
  API_BEGIN
  auto cp = [](int32_t *dst, const std::vector<int32_t> &v) { if (dst && !v.empty()) std::memcpy(dst, v.data(), v.size() * 4); };
  cp(face_parent, m->f_parent); cp(face_neighbor, m->f_neighbor); cp(face_bc, m->f_bc); cp(face_nodes, m->f_nodes);
  cp(cell_face_index, m->cf_index); cp(cell_faces, m->cf_list); cp(nbr_index, m->nbr_index); cp(nbrs, m->nbr_list);
  cp(grad_index, m->st_index); cp(grad_keys, m->st_keys);
  API_END
}

int fcfd_mesh_geometry(const fcfd_mesh *m, double *face_normal, double *face_area, double *face_centroid,
                       double *face_avg, double *cell_centroid, double *cell_volume, double *cell_length,
                       double *cell_wall_distance, double *length_scale) {
  API_BEGIN
  auto cp = [](double *dst, const std::vector<double> &v) { if (dst && !v.empty()) std::memcpy(dst, v.data(), v.size() * 8); };
  cp(face_normal, m->f_normal); cp(face_area, m->f_area); cp(face_centroid, m->f_centroid); cp(face_avg, m->f_w);
  cp(cell_centroid, m->c_centroid); cp(cell_volume, m->c_volume); cp(cell_length, m->c_length); cp(cell_wall_distance, m->c_wall);
  if (length_scale) *length_scale = m->length_scale;
  API_END
}

int fcfd_mesh_lsq(const fcfd_mesh *m, double *cofactors, double *self_weight) {
  API_BEGIN
  if (cofactors) std::memcpy(cofactors, m->st_cof.data(), m->st_cof.size() * 8);
  if (self_weight) std::memcpy(self_weight, m->st_self.data(), m->st_self.size() * 8);
  API_END
}

int fcfd_mesh_grad_weights(const fcfd_mesh *m, double *weights) {
  API_BEGIN
  if (!m || !weights) throw Error(FCFD_ERR_INPUT, "null argument");
  if (!m->grad_weights) throw Error(FCFD_ERR_UNSUPPORTED, "the mesh keeps no stored gradient weights (no curvilinear cell)");
  std::memcpy(weights, m->st_w.data(), m->st_w.size() * sizeof(double));
  API_END
}

int fcfd_mesh_rcm(const fcfd_mesh *m, int32_t *perm) {
  API_BEGIN
  if (!m || !perm) throw Error(FCFD_ERR_INPUT, "null argument");
  std::vector<int32_t> p;
  rcm_order(*m, p);
  std::memcpy(perm, p.data(), sizeof(int32_t) * p.size());
  API_END
}

int fcfd_ctx_create(const fcfd_mesh *mp, const fcfd_case *csp, int device, fcfd_ctx **out) {
  API_BEGIN
  if (!mp || !csp || !out) throw Error(FCFD_ERR_INPUT, "null argument");
  const fcfd_mesh &m = *mp;
  const fcfd_case &c = *csp;
  if ((int)c.bc.size() > kMaxBC) throw Error(FCFD_ERR_UNSUPPORTED, "more than 16 boundary regions");
  for (const BcRegion &b : c.bc)
    if (b.type == BC_OUTLET && b.specified == SP_STATE)
      throw Error(FCFD_ERR_INPUT, "you can't specify complete thermodynamic state at an outlet");
  std::unique_ptr<fcfd_ctx> x(new fcfd_ctx());
  x->device = device;
  CK(cudaSetDevice(device));
  CK(cudaStreamCreateWithFlags(&x->stream, cudaStreamNonBlocking));
  CK(cudaStreamCreateWithFlags(&x->side, cudaStreamNonBlocking));
  CK(cudaEventCreateWithFlags(&x->ev_fork, cudaEventDisableTiming));
  CK(cudaEventCreateWithFlags(&x->ev_join, cudaEventDisableTiming));
  x->mesh = mp;
  x->case_ptr = csp;
  DevCase &d = x->cs;
  const Material &mt = c.mat;
  d.gamma = mt.gamma; d.R = mt.R; d.Pref = mt.Pref; d.Tref = mt.Tref; d.Minf = c.Minf; d.K = c.limiter_threshold;
  d.Lref = m.length_scale; d.Cp = mt.Cp(); d.mu = mt.mu; d.lambda = mt.lambda; d.sut_mu_ref = mt.sut_mu_ref;
  d.sut_T_ref = mt.sut_T_ref; d.sut_S = mt.sut_S; d.Pr = mt.Pr; d.Pr_t = c.Pr_t; d.sutherland = mt.sutherland;
  d.prandtl = mt.prandtl; d.flux = c.flux; d.limiter = c.limiter; d.order = c.order; d.nbc = (int)c.bc.size();
  d.wdiss = c.wdiss; d.bl_height = c.bl_height;
  bool fixed_q = false;
  for (size_t b = 0; b < c.bc.size(); ++b) {
    const BcRegion &r = c.bc[b];
    DevBC &o = d.bc[b];
    o.type = r.type; o.kind = r.kind; o.specified = r.specified; o.thermal = r.thermal;
    o.p = r.p; o.T = r.T; o.rho = r.rho; o.qdot = r.qdot; o.p_total = r.p_total; o.T_total = r.T_total;
    o.mdot_per_area = r.mdot / m.bc_total_area[b];
    for (int k = 0; k < 3; ++k) o.V[k] = r.V[k];
    o.T_fixed = r.T_fixed ? 1 : 0;
    o.p_fixed = r.p_fixed ? 1 : 0;
    o.V_fixed = r.V_fixed ? 1 : 0;
    if (r.thermal == TH_FIXED_Q && r.type == BC_WALL) fixed_q = true;
  }
  x->viscous = mt.sutherland || mt.prandtl || mt.mu != 0. || mt.lambda != 0. || fixed_q;
  d.viscous = x->viscous;
  // Limiters that are continuous in the gradient take the fused (non bit-exact)
  // gradient; minmod, Barth-Jespersen and VK with K = 0 decide on the sign of
  // rounding noise and take the bit-exact one.
  d.fast_grad = (c.order == ORDER_FIRST || c.limiter == LIM_NONE || (c.limiter == LIM_VK && c.limiter_threshold > 0.)) ? 1 : 0;
  // ---- mesh upload (SoA)
  const int nc = m.nc, nf = m.nf, nb = m.nb, nt = nc + nb;
  x->f_parent.upload(m.f_parent); x->f_neighbor.upload(m.f_neighbor); x->f_bc.upload(m.f_bc);
  x->f_n.upload(soa(m.f_normal, nf, 3)); x->f_area.upload(m.f_area); x->f_x.upload(soa(m.f_centroid, nf, 3));
  x->f_w.upload(soa(m.f_w, nf, 2)); x->c_x.upload(soa(m.c_centroid, nt, 3));
  std::vector<double> clen(m.c_length.begin(), m.c_length.begin() + nc);
  x->c_len.upload(clen);
  x->cf_index.upload(m.cf_index);
  std::vector<int32_t> cfl(m.cf_list.size());
  for (int cc = 0; cc < nc; ++cc)
    for (int j = m.cf_index[cc]; j < m.cf_index[cc + 1]; ++j) {
      int f = m.cf_list[j];
      cfl[j] = (m.f_parent[f] == cc) ? f : ~f;
    }
  x->cf_list.upload(cfl);
  x->st_index.upload(m.st_index); x->st_keys.upload(m.st_keys);
  x->st_cof.upload(soa(m.st_cof, nc, 7)); x->st_self.upload(soa(m.st_self, nc, 3));
  x->st_recip.upload(m.st_recip); x->st_mirror.upload(soa(m.st_mirror, nc, 3));
  if (m.grad_weights) {
    // stored map weights (a curvilinear case): the gradient sums them in key
    // order; the fused and two-warp least-squares forms do not apply
    x->st_w.upload(m.st_w);
    d.fast_grad = 0;
  }
  if (c.flux == FLUX_SW) {
    if ((int)m.f_wall.size() != nf || (int)m.f_diss.size() != nf)
      throw Error(FCFD_ERR_INPUT, "the Steger-Warming flux needs a mesh built with a Steger-Warming case (face wall distances)");
    x->f_wall.upload(m.f_wall); x->f_diss.upload(m.f_diss);
  }
  {
    std::vector<double> vol(m.c_volume.begin(), m.c_volume.begin() + nc);
    x->c_vol.upload(vol);
    for (int cc = 0; cc < nc; ++cc)
      if (m.st_index[cc] == m.st_index[cc + 1]) { x->green_gauss = true; break; }
  }
  d.pair_grad = (x->green_gauss || m.grad_weights) ? 0 : 1;
  if (!x->green_gauss && !m.grad_weights) {
    // tiles of kGradTile consecutive cells for the shared-memory gradient
    // kernel: each tile's staged set (the cells its stencils and faces name,
    // ascending) and every stencil / face entry as a slot in it
    const int T = kGradTile, ntile = (nc + T - 1) / T;
    std::vector<int32_t> toff(ntile + 1, 0), tcells, stl(m.st_keys.size()), cfl_loc(m.cf_list.size()), selfl(nc);
    std::vector<int32_t> set;
    int smax = 0;
    for (int t = 0; t < ntile; ++t) {
      const int c0 = t * T, c1 = std::min(nc, c0 + T);
      set.clear();
      for (int c = c0; c < c1; ++c) {
        for (int j = m.st_index[c]; j < m.st_index[c + 1]; ++j) set.push_back(m.st_keys[j]);
        for (int j = m.cf_index[c]; j < m.cf_index[c + 1]; ++j) {
          const int f = m.cf_list[j];
          set.push_back(m.f_parent[f] == c ? m.f_neighbor[f] : m.f_parent[f]);
        }
        set.push_back(c);
      }
      std::sort(set.begin(), set.end());
      set.erase(std::unique(set.begin(), set.end()), set.end());
      auto slot = [&](int k) { return (int32_t)(std::lower_bound(set.begin(), set.end(), k) - set.begin()); };
      for (int c = c0; c < c1; ++c) {
        selfl[c] = slot(c);
        for (int j = m.st_index[c]; j < m.st_index[c + 1]; ++j) stl[j] = slot(m.st_keys[j]);
        for (int j = m.cf_index[c]; j < m.cf_index[c + 1]; ++j) {
          const int f = m.cf_list[j];
          cfl_loc[j] = slot(m.f_parent[f] == c ? m.f_neighbor[f] : m.f_parent[f]);
        }
      }
      tcells.insert(tcells.end(), set.begin(), set.end());
      toff[t + 1] = (int32_t)tcells.size();
      smax = std::max(smax, (int)set.size());
    }
    int optin = 0;
    CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
    const size_t smem = sizeof(double) * 8 * (size_t)smax;
    if (smem <= (size_t)optin) {
      x->tile_off.upload(toff); x->tile_cells.upload(tcells); x->st_local.upload(stl);
      x->cf_local.upload(cfl_loc); x->self_local.upload(selfl);
      x->dm.tile_slots_max = smax;
      CK(cudaFuncSetAttribute(k_grad_limiter_tile<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      CK(cudaFuncSetAttribute(k_grad_limiter_tile<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    }
  }
  d.tile_grad = 0;
  d.fold_grad = 0;
  if (!x->green_gauss && !m.grad_weights) {
    // Folded stencils for the fused gradient (kind 3): a ghost of a symmetry face whose
    // normal is exactly (0, 0, +-1) holds its parent's state with w negated
    // (the symmetry branch of apply_bc), so where the parent is in the same
    // stencil the ghost's term w (phi_g - phi_c) d joins the parent's entry.
    // Built when folding removes at least a third of the entries (extruded
    // one-layer meshes: 27 entries become 9).
    std::vector<int32_t> gh_face(nb, -1);  // ghost nc + g is the neighbour of boundary face gh_face[g]
    for (int f = 0; f < nf; ++f)
      if (m.f_bc[f] >= 0) gh_face[m.f_neighbor[f] - nc] = f;
    auto zsym = [&](int k) {
      if (k < nc) return -1;
      const int f = gh_face[k - nc];
      const BcRegion &br = c.bc[m.f_bc[f]];
      if (br.type != BC_SYMMETRY) return -1;
      if (m.f_normal[3 * (size_t)f] != 0. || m.f_normal[3 * (size_t)f + 1] != 0.) return -1;
      return m.f_parent[f];
    };
    std::vector<int32_t> fidx(nc + 1, 0), fkey;
    std::vector<double> fe;
    std::vector<int32_t> keys;
    for (int cc = 0; cc < nc; ++cc) {
      const double xc0 = m.c_centroid[3 * (size_t)cc], xc1 = m.c_centroid[3 * (size_t)cc + 1], xc2 = m.c_centroid[3 * (size_t)cc + 2];
      const int j0 = m.st_index[cc], j1 = m.st_index[cc + 1];
      keys.assign(m.st_keys.begin() + j0, m.st_keys.begin() + j1);
      const size_t e0 = fkey.size();
      auto slot = [&](int k) -> size_t {
        for (size_t q = e0; q < fkey.size(); ++q)
          if (fkey[q] == k) return q;
        fkey.push_back(k);
        for (int t = 0; t < 6; ++t) fe.push_back(0.);
        return fkey.size() - 1;
      };
      for (int k : keys) {
        const double d0 = m.c_centroid[3 * (size_t)k] - xc0, d1 = m.c_centroid[3 * (size_t)k + 1] - xc1,
                     d2 = m.c_centroid[3 * (size_t)k + 2] - xc2;
        const double w = d0 * d0 + d1 * d1 + d2 * d2;
        const int par = zsym(k);
        const bool folded = par >= 0 && std::find(keys.begin(), keys.end(), par) != keys.end();
        if (k == cc) { slot(cc); continue; }  // the self entry contributes nothing
        const size_t q = slot(folded ? par : k);
        const int o = folded ? 3 : 0;
        fe[6 * q + o] += w * d0; fe[6 * q + o + 1] += w * d1; fe[6 * q + o + 2] += w * d2;
      }
      fidx[cc + 1] = (int32_t)fkey.size();
    }
    if (3 * fkey.size() <= 2 * m.st_keys.size()) {
      x->fold_index.upload(fidx); x->fold_key.upload(fkey); x->fold_e.upload(fe);
    }
  }
  std::vector<int32_t> bface(nb), outl;
  for (int f = 0; f < nf; ++f) {
    if (m.f_bc[f] >= 0) {
      bface[m.f_neighbor[f] - nc] = f;
      if (c.bc[m.f_bc[f]].type == BC_OUTLET) outl.push_back(f);
    }
  }
  x->bface.upload(bface);
  {
    // main face launch order: blocks of 4096 parent cells; within a block the
    // interior faces, then each BC region's faces (face order within a
    // group), so that a warp's faces take one branch and a boundary face
    // reads its parent's state, gradients and limiters while the block's
    // interior faces have them in L2.  Meshes whose cell data L2 holds whole
    // (under 148 x 512 cells) keep one block: the measured cylinder 256x128
    // face kernel was 0.6 us slower with blocks.
    std::vector<int32_t> order(nf);
    for (int f = 0; f < nf; ++f) order[f] = f;
    const int blk_shift = nc < kPairGradCells ? 30 : 12;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
      const int ba = m.f_parent[a] >> blk_shift, bb = m.f_parent[b] >> blk_shift;
      return ba != bb ? ba < bb : m.f_bc[a] < m.f_bc[b];
    });
    x->face_order.upload(order);
  }
  x->color_cells.upload(m.color_cells);
  x->color_index = m.color_index;
  {
    // packed Gauss-Seidel couplings (colour by colour, slot-major)
    const std::vector<int> &ci = m.color_index;
    const std::vector<int> &cc = m.color_cells;
    int deg = 0;
    for (int c = 0; c < nc; ++c) {
      int d = 0;
      for (int j = m.cf_index[c]; j < m.cf_index[c + 1]; ++j) {
        if (m.f_bc[m.cf_list[j]] < 0) ++d;
      }
      deg = std::max(deg, d);
    }
    std::vector<int> nbr((size_t)nc * deg, -1), src((size_t)nc * deg, 0);
    for (size_t col = 0; col + 1 < ci.size(); ++col) {
      const int base = ci[col], cnt = ci[col + 1] - ci[col];
      for (int i = 0; i < cnt; ++i) {
        const int c = cc[base + i];
        int slot = 0;
        for (int j = m.cf_index[c]; j < m.cf_index[c + 1]; ++j) {
          // host cf_list holds plain face indices; src is signed like the
          // device list (~f where this cell is the face's neighbour)
          const int f = m.cf_list[j];
          if (m.f_bc[f] >= 0) continue;
          const bool parent = m.f_parent[f] == c;
          const size_t at = (size_t)base * deg + (size_t)slot * cnt + i;
          nbr[at] = parent ? m.f_neighbor[f] : m.f_parent[f];
          src[at] = parent ? f : ~f;
          ++slot;
        }
      }
    }
    x->gs_deg = deg;
    if (deg > 0) { x->gs_nbr.upload(nbr); x->gs_src.upload(src); }
  }
  x->outlet.upload(outl);
  x->n_outlet = (int)outl.size();
  // ---- state buffers
  x->p64.alloc(nc, nf, nb);
  x->Win.alloc(5 * (size_t)nc); x->Vin.alloc(5 * (size_t)nc); x->Rtmp.alloc(5 * (size_t)nc); x->dt.alloc(nc);
  x->mdot.alloc(nf); x->wl.alloc(nf); x->ext.alloc(8); x->err.alloc(1); x->argx.alloc(8); x->dtmin.alloc(1);
  CK(cudaMemset(x->err.p, 0, sizeof(int)));
  {
    // arm the extrema slots (max slots start at key 0, min slots at all
    // ones) and the first-attaining-cell slots; every residual chain's gather
    // re-arms them for the next chain
    unsigned long long e0[8];
    int a0[8];
    for (int k = 0; k < 8; ++k) { e0[k] = (k & 1) ? ~0ull : 0ull; a0[k] = 0x7F7F7F7F; }
    CK(cudaMemcpy(x->ext.p, e0, sizeof(e0), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(x->argx.p, a0, sizeof(a0), cudaMemcpyHostToDevice));
  }
  DevMesh &dm = x->dm;
  dm.nc = nc; dm.nf = nf; dm.nb = nb; dm.nt = nt;
  dm.f_parent = x->f_parent.p; dm.f_neighbor = x->f_neighbor.p; dm.f_bc = x->f_bc.p;
  dm.f_n = x->f_n.p; dm.f_area = x->f_area.p; dm.f_x = x->f_x.p; dm.f_w = x->f_w.p; dm.c_x = x->c_x.p;
  dm.c_len = x->c_len.p; dm.cf_index = x->cf_index.p; dm.cf_list = x->cf_list.p; dm.st_index = x->st_index.p;
  dm.st_keys = x->st_keys.p; dm.st_cof = x->st_cof.p; dm.st_self = x->st_self.p; dm.bface = x->bface.p;
  dm.st_recip = x->st_recip.p; dm.st_mirror = x->st_mirror.p; dm.c_vol = x->c_vol.p;
  dm.st_w = x->st_w.p;
  dm.tile_off = x->tile_off.p; dm.tile_cells = x->tile_cells.p; dm.st_local = x->st_local.p;
  dm.cf_local = x->cf_local.p; dm.self_local = x->self_local.p;
  dm.fold_index = x->fold_index.p; dm.fold_key = x->fold_key.p; dm.fold_e = x->fold_e.p;
  dm.f_wall = x->f_wall.p; dm.f_diss = x->f_diss.p;
  dm.outlet_faces = x->outlet.p; dm.n_outlet = x->n_outlet;
  dm.face_list = x->face_order.p; dm.n_face_list = nf;
  rans_setup(x.get());  // k-omega BC values and buffers (turbulent cases only)
  CK(cudaDeviceSynchronize());
  *out = x.release();
  API_END
}

void fcfd_ctx_destroy(fcfd_ctx *x) {
  if (!x) return;
  cudaSetDevice(x->device);
  if (x->graph) cudaGraphExecDestroy(x->graph);
  if (x->host_graph) cudaGraphExecDestroy(x->host_graph);
  if (x->err_pinned) cudaFreeHost(x->err_pinned);
  adjoint_free(x);
  rans_free(x);
  if (x->ev_fork) cudaEventDestroy(x->ev_fork);
  if (x->ev_join) cudaEventDestroy(x->ev_join);
  if (x->side) cudaStreamDestroy(x->side);
  if (x->stream) cudaStreamDestroy(x->stream);
  delete x;
}

// page-locked (pinned or registered) host memory
static bool host_pinned(const void *p) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

int fcfd_residual(fcfd_ctx *x, const double *W, double *R, int flags) {
  API_BEGIN
  if (!x || !W || !R) throw Error(FCFD_ERR_INPUT, "null argument");
  CK(cudaSetDevice(x->device));
  const DevMesh &m = x->dm;
  const bool dev = flags & FCFD_DEVICE_PTRS;
  if (!dev && host_pinned(W) && host_pinned(R)) {
    // one graph launch: host-to-device copy, the chain, device-to-host copy
    // and the error flag, then one synchronisation
    cudaStream_t s = x->stream;
    if (!x->err_pinned) CK(cudaMallocHost((void **)&x->err_pinned, sizeof(int)));
    if (!x->host_graph || x->host_graph_W != W || x->host_graph_R != R || x->host_graph_fast_grad != x->cs.fast_grad) {
      if (x->host_graph) { CK(cudaGraphExecDestroy(x->host_graph)); x->host_graph = nullptr; }
      cudaGraph_t g = nullptr;
      CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
      CK(cudaMemcpyAsync(x->Win.p, W, sizeof(double) * 5 * m.nc, cudaMemcpyHostToDevice, s));
      k_aos_to_soa<double><<<(m.nc + 255) / 256, 256, 0, s>>>(x->Win.p, x->p64.W.p, m.nc, m.nt);
      launch_chain<double>(x, x->p64, x->Rtmp.p, true, x->mdot.p, x->wl.p);
      CK(cudaMemcpyAsync(R, x->Rtmp.p, sizeof(double) * 5 * m.nc, cudaMemcpyDeviceToHost, s));
      CK(cudaMemcpyAsync(x->err_pinned, x->err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
      CK(cudaStreamEndCapture(s, &g));
      CK(cudaGraphInstantiate(&x->host_graph, g, 0));
      CK(cudaGraphDestroy(g));
      x->host_graph_W = W;
      x->host_graph_R = R;
      x->host_graph_fast_grad = x->cs.fast_grad;
    }
    CK(cudaGraphLaunch(x->host_graph, s));
    CK(cudaStreamSynchronize(s));
    if (*x->err_pinned) check_err(x);  // reports and clears the flag
    return FCFD_OK;
  }
  const double *win = W;
  if (!dev) {
    CK(cudaMemcpyAsync(x->Win.p, W, sizeof(double) * 5 * m.nc, cudaMemcpyHostToDevice, x->stream));
    win = x->Win.p;
  }
  k_aos_to_soa<double><<<(m.nc + 255) / 256, 256, 0, x->stream>>>(win, x->p64.W.p, m.nc, m.nt);
  double *rout = dev ? R : x->Rtmp.p;
  launch_chain<double>(x, x->p64, rout, true, x->mdot.p, x->wl.p);
  if (!dev) CK(cudaMemcpyAsync(R, x->Rtmp.p, sizeof(double) * 5 * m.nc, cudaMemcpyDeviceToHost, x->stream));
  check_err(x);
  API_END
}

int fcfd_last_stages(fcfd_ctx *x, double *grads, double *limiter, double *ghost, double *mdot, double *weightL) {
  API_BEGIN
  CK(cudaSetDevice(x->device));
  CK(cudaStreamSynchronize(x->stream));
  const DevMesh &m = x->dm;
  auto get = [&](const double *src, size_t n, int k, double *dst) {
    if (!dst) return;
    std::vector<double> h(n * k);
    CK(cudaMemcpy(h.data(), src, sizeof(double) * n * k, cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < n; ++i)
      for (int j = 0; j < k; ++j) dst[i * k + j] = h[j * n + i];
  };
  get(x->p64.G.p, m.nc, 15, grads);
  get(x->p64.Lm.p, m.nc, 5, limiter);
  if (ghost) {
    std::vector<double> h(5 * (size_t)m.nt);
    CK(cudaMemcpy(h.data(), x->p64.W.p, sizeof(double) * 5 * m.nt, cudaMemcpyDeviceToHost));
    for (int g = 0; g < m.nb; ++g)
      for (int v = 0; v < 5; ++v) ghost[5 * g + v] = h[(size_t)v * m.nt + m.nc + g];
  }
  if (mdot) CK(cudaMemcpy(mdot, x->mdot.p, sizeof(double) * m.nf, cudaMemcpyDeviceToHost));
  if (weightL) CK(cudaMemcpy(weightL, x->wl.p, sizeof(double) * m.nf, cudaMemcpyDeviceToHost));
  API_END
}

int fcfd_local_dt(fcfd_ctx *x, const double *W, double cfl, int mode, double *dt, int flags) {
  API_BEGIN
  CK(cudaSetDevice(x->device));
  const DevMesh &m = x->dm;
  const bool dev = flags & FCFD_DEVICE_PTRS;
  const double *win = W;
  if (!dev) {
    CK(cudaMemcpyAsync(x->Win.p, W, sizeof(double) * 5 * m.nc, cudaMemcpyHostToDevice, x->stream));
    win = x->Win.p;
  }
  k_aos_to_soa<double><<<(m.nc + 255) / 256, 256, 0, x->stream>>>(win, x->p64.W.p, m.nc, m.nt);
  double *out = dev ? dt : x->dt.p;
  if (mode == 1) CK(cudaMemsetAsync(x->dtmin.p, 0xFF, sizeof(unsigned long long), x->stream));
  k_local_dt<double><<<(m.nc + 255) / 256, 256, 0, x->stream>>>(x->cs, m, x->p64.W.p, out, cfl, mode == 1 ? x->dtmin.p : nullptr);
  if (mode == 1) k_fill_min<double><<<(m.nc + 255) / 256, 256, 0, x->stream>>>(m.nc, out, x->dtmin.p);
  CK(cudaGetLastError());
  if (!dev) CK(cudaMemcpyAsync(dt, x->dt.p, sizeof(double) * m.nc, cudaMemcpyDeviceToHost, x->stream));
  CK(cudaStreamSynchronize(x->stream));
  API_END
}

// out[0] = average ms per residual: the whole chain (ghost states + extrema,
// gradient + limiter, face flux with the stale outlet densities, gather),
// replayed as one CUDA graph between two CUDA events on the context stream;
// out[1..5] = per-kernel averages from a second pass with an event after
// every kernel: ghost+extrema, gradient+limiter, (unused: the outlet density
// is computed inside the face flux), face flux, gather.  L2 is flushed (a
// 512 MB memset) before every residual when flush_l2 is set.
int fcfd_residual_mixed(fcfd_ctx *x, const double *W, double *R, double shock_ratio, int32_t flags,
                        int64_t *n_fp64_faces) {
  API_BEGIN
  if (!x || !W || !R) throw Error(FCFD_ERR_INPUT, "null argument");
  if (!(shock_ratio == shock_ratio)) throw Error(FCFD_ERR_INPUT, "shock_ratio is NaN");
  CK(cudaSetDevice(x->device));
  const DevMesh &m = x->dm;
  cudaStream_t s = x->stream;
  const bool dev = flags & FCFD_DEVICE_PTRS;
  const double *win = W;
  if (!dev) {
    CK(cudaMemcpyAsync(x->Win.p, W, sizeof(double) * 5 * m.nc, cudaMemcpyHostToDevice, s));
    win = x->Win.p;
  }
  k_aos_to_soa<double><<<(m.nc + 255) / 256, 256, 0, s>>>(win, x->p64.W.p, m.nc, m.nt);
  double *rout = dev ? R : x->Rtmp.p;
  launch_mixed(x, shock_ratio, rout);
  if (!dev) CK(cudaMemcpyAsync(R, x->Rtmp.p, sizeof(double) * 5 * m.nc, cudaMemcpyDeviceToHost, s));
  int cnt = 0;
  CK(cudaMemcpyAsync(&cnt, x->mx_count.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  if (n_fp64_faces) *n_fp64_faces = cnt;
  check_err(x);
  API_END
}

int fcfd_time_residual_mixed(fcfd_ctx *x, int32_t reps, int32_t flush_l2, double shock_ratio, double *out) {
  API_BEGIN
  if (!x || !out || reps < 1) throw Error(FCFD_ERR_INPUT, "bad argument");
  CK(cudaSetDevice(x->device));
  cudaStream_t s = x->stream;
  if (flush_l2 && x->flush.n == 0) x->flush.alloc((size_t)512 << 20);
  Timing t;
  double acc = 0.;
  for (int r = 0; r < reps; ++r) {
    if (flush_l2) CK(cudaMemsetAsync(x->flush.p, r & 0xff, x->flush.n, s));
    CK(cudaEventRecord(t.ev[0], s));
    launch_mixed(x, shock_ratio, x->p64.R.p);
    CK(cudaEventRecord(t.ev[1], s));
    CK(cudaEventSynchronize(t.ev[1]));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, t.ev[0], t.ev[1]));
    acc += ms;
  }
  int cnt = 0;
  CK(cudaMemcpyAsync(&cnt, x->mx_count.p, sizeof(int), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  out[0] = acc / reps;
  out[1] = cnt;
  check_err(x);
  API_END
}

int fcfd_time_residual(fcfd_ctx *x, int reps, int flush_l2, double *out, int out_len) {
  API_BEGIN
  CK(cudaSetDevice(x->device));
  const DevMesh &m = x->dm;
  cudaStream_t s = x->stream;
  if (flush_l2 && x->flush.n == 0) x->flush.alloc((size_t)512 << 20);
  Timing t;
  double acc[6] = {0, 0, 0, 0, 0, 0};
  const int tb = 256;
  Pipe<double> &P = x->p64;
  const bool need_ext = x->cs.limiter == 1 && x->cs.order != 1;
  const int ng = (m.nb + tb - 1) / tb + (need_ext ? kExtremaBlocks : 0);
  auto kernel = [&](int k) {
    if (k == 0) {
      if (ng > 0) k_ghost_minmax<double><<<ng, tb, 0, s>>>(x->cs, m, P.W.p, need_ext ? x->ext.p : nullptr, x->err.p);
    } else if (k == 1) {
      launch_grad_limiter<double>(x->cs, m, P.W.p, x->ext.p, nullptr, P.G.p, P.Lm.p, s, x->pdl);
    } else if (k == 3) {
      launch_faces<double>(x, P, nullptr, nullptr, nullptr, s);
    } else if (k == 4) {
      k_gather<double, false><<<(5 * m.nc + tb - 1) / tb, tb, 0, s>>>(m, P.D.p, P.R.p, x->ext.p, x->argx.p);
    }
  };
  // the chain as one CUDA graph (captured once per context and case
  // settings), replayed between the two events
  if (!x->graph || x->graph_fast_grad != x->cs.fast_grad) {
    if (x->graph) { cudaGraphExecDestroy(x->graph); x->graph = nullptr; }
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    for (int k = 0; k < 5; ++k) kernel(k);
    CK(cudaStreamEndCapture(s, &g));
    CK(cudaGraphInstantiate(&x->graph, g, 0));
    CK(cudaGraphDestroy(g));
    x->graph_fast_grad = x->cs.fast_grad;
  }
  for (int r = 0; r < reps; ++r) {
    if (flush_l2) CK(cudaMemsetAsync(x->flush.p, r & 0xff, x->flush.n, s));
    CK(cudaEventRecord(t.ev[0], s));
    CK(cudaGraphLaunch(x->graph, s));
    CK(cudaEventRecord(t.ev[5], s));
    CK(cudaGetLastError());
    CK(cudaEventSynchronize(t.ev[5]));
    float ms;
    CK(cudaEventElapsedTime(&ms, t.ev[0], t.ev[5]));
    acc[0] += ms;
  }
  for (int r = 0; r < reps; ++r) {
    if (flush_l2) CK(cudaMemsetAsync(x->flush.p, r & 0xff, x->flush.n, s));
    CK(cudaEventRecord(t.ev[0], s));
    for (int k = 0; k < 5; ++k) {
      kernel(k);
      CK(cudaEventRecord(t.ev[k + 1], s));
    }
    CK(cudaGetLastError());
    CK(cudaEventSynchronize(t.ev[5]));
    float ms;
    for (int k = 0; k < 5; ++k) { CK(cudaEventElapsedTime(&ms, t.ev[k], t.ev[k + 1])); acc[k + 1] += ms; }
  }
  for (int k = 0; k < 6 && k < out_len; ++k) out[k] = acc[k] / reps;
  API_END
}

int fcfd_ctx_set_gradient_kernel(fcfd_ctx *x, int kind) {
  API_BEGIN
  if (!x) throw Error(FCFD_ERR_INPUT, "null context");
  if (kind < 0 || kind > 3) throw Error(FCFD_ERR_INPUT, "gradient kernel kind must be 0, 1, 2 or 3");
  if (kind == 2 && !x->dm.tile_off) throw Error(FCFD_ERR_UNSUPPORTED, "no gradient tiles for this mesh (Green-Gauss or curvilinear cells, or a tile's cells exceed shared memory)");
  if (kind == 3 && !x->dm.fold_index) throw Error(FCFD_ERR_UNSUPPORTED, "no folded stencils for this mesh (fewer than a third of the entries are z-symmetry ghosts of stencil cells)");
  x->grad_kernel = kind;
  x->cs.tile_grad = (kind == 2) ? 1 : 0;
  x->cs.fold_grad = (kind == 3) ? 1 : 0;
  // the captured chains hold the previous gradient kernel
  if (x->graph) { CK(cudaGraphExecDestroy(x->graph)); x->graph = nullptr; }
  if (x->host_graph) { CK(cudaGraphExecDestroy(x->host_graph)); x->host_graph = nullptr; }
  API_END
}

int fcfd_ctx_set_launch_overlap(fcfd_ctx *x, int32_t on) {
  API_BEGIN
  if (!x) throw Error(FCFD_ERR_INPUT, "null context");
  x->pdl = on != 0;
  if (x->graph) { CK(cudaGraphExecDestroy(x->graph)); x->graph = nullptr; }
  if (x->host_graph) { CK(cudaGraphExecDestroy(x->host_graph)); x->host_graph = nullptr; }
  API_END
}

int fcfd_ctx_gradient_info(const fcfd_ctx *x, int64_t *out) {
  API_BEGIN
  if (!x || !out) throw Error(FCFD_ERR_INPUT, "null argument");
  out[0] = x->cs.tile_grad ? 2 : ((x->cs.fold_grad && x->cs.fast_grad) ? 3 : 1);
  out[1] = (int64_t)x->fold_key.n;
  out[2] = x->cs.fast_grad;
  API_END
}

int fcfd_ctx_set_exact_gradients(fcfd_ctx *x, int exact) {
  API_BEGIN
  if (!x) throw Error(FCFD_ERR_INPUT, "null context");
  if (exact || x->dm.st_w) x->cs.fast_grad = 0;
  else {
    const fcfd_case *c = x->case_ptr;
    x->cs.fast_grad = (c->order == ORDER_FIRST || c->limiter == LIM_NONE || (c->limiter == LIM_VK && c->limiter_threshold > 0.)) ? 1 : 0;
  }
  API_END
}

// Forward tangent: JV = dR/dW . V (and R if requested).
int fcfd_jvp(fcfd_ctx *x, const double *W, const double *V, double *R, double *JV, int flags) {
  API_BEGIN
  if (!x || !W || !V || !JV) throw Error(FCFD_ERR_INPUT, "null argument");
  CK(cudaSetDevice(x->device));
  const DevMesh &m = x->dm;
  const bool dev = flags & FCFD_DEVICE_PTRS;
  const bool f32 = flags & FCFD_JVP_FP32;
  if (!f32 && !x->pjv.ready) x->pjv.alloc(m.nc, m.nf, m.nb);
  if (f32 && !x->pjv32.ready) x->pjv32.alloc(m.nc, m.nf, m.nb);
  const double *w = W, *v = V;
  if (!dev) {
    CK(cudaMemcpyAsync(x->Win.p, W, sizeof(double) * 5 * m.nc, cudaMemcpyHostToDevice, x->stream));
    CK(cudaMemcpyAsync(x->Vin.p, V, sizeof(double) * 5 * m.nc, cudaMemcpyHostToDevice, x->stream));
    w = x->Win.p; v = x->Vin.p;
  }
  double *rout = R ? (dev ? R : x->Rtmp.p) : nullptr;
  double *jout = dev ? JV : x->Vin.p;
  if (f32) {
    k_seed_dual<float><<<(m.nc + 255) / 256, 256, 0, x->stream>>>(w, v, x->pjv32.W.p, m.nc, m.nt);
    launch_chain<Dual<float>>(x, x->pjv32, x->pjv32.R.p, false, nullptr, nullptr);
    k_split_dual<float><<<(m.nc + 255) / 256, 256, 0, x->stream>>>(x->pjv32.R.p, rout, jout, m.nc);
  } else {
    k_seed_dual<double><<<(m.nc + 255) / 256, 256, 0, x->stream>>>(w, v, x->pjv.W.p, m.nc, m.nt);
    launch_chain<Dual<double>>(x, x->pjv, x->pjv.R.p, false, nullptr, nullptr);
    k_split_dual<double><<<(m.nc + 255) / 256, 256, 0, x->stream>>>(x->pjv.R.p, rout, jout, m.nc);
  }
  CK(cudaGetLastError());
  if (!dev) {
    if (R) CK(cudaMemcpyAsync(R, x->Rtmp.p, sizeof(double) * 5 * m.nc, cudaMemcpyDeviceToHost, x->stream));
    CK(cudaMemcpyAsync(JV, x->Vin.p, sizeof(double) * 5 * m.nc, cudaMemcpyDeviceToHost, x->stream));
  }
  check_err(x);
  API_END
}

int fcfd_point_flux(int flux, const double *L, const double *R, const double *n, double gamma, double gas_R, double Pref,
                    double Tref, double Minf, double *out, double *weightL) {
  API_BEGIN
  DevCase c{};
  c.gamma = gamma; c.R = gas_R; c.Pref = Pref; c.Tref = Tref; c.Minf = Minf;
  FState<double> a{}, b{};
  a.p = L[0]; a.V[0] = L[1]; a.V[1] = L[2]; a.V[2] = L[3]; a.T = L[4];
  b.p = R[0]; b.V[0] = R[1]; b.V[1] = R[2]; b.V[2] = R[3]; b.T = R[4];
  a.rho = eos_rho(c, a.p, a.T); b.rho = eos_rho(c, b.p, b.T);
  finish(c, a, n); finish(c, b, n);
  double F[5], wl = 0;
  if (flux == FLUX_ROE) roe(c, a, b, n, F, wl);
  else if (flux == FLUX_VAN_LEER) vanleer(c, a, b, n, F, wl);
  else if (flux == FLUX_AUSM_PLUS_UP) ausm(c, a, b, n, F, wl);
  else if (flux == FLUX_SD_SLAU) sdslau(c, a, b, n, F, wl);
  else throw Error(FCFD_ERR_UNSUPPORTED, "point flux: 1 Roe, 2 Van Leer, 3 AUSM+up, 4 SD-SLAU (Steger-Warming needs face wall data)");
  for (int k = 0; k < 5; ++k) out[k] = F[k];
  if (weightL) *weightL = wl;
  API_END
}

}  // extern "C"
