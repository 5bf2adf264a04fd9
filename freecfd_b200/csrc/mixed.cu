// Mixed-precision residual: the face pass in FP32, FP64 at shocks.
//
// The residual of ns_assemble_linear_system.cc:75-140 with the same ghost
// update, gradients and limiters as the FP64 chain (FP64: on one-layer meshes
// the reference's minmod / Barth-Jespersen decisions follow the sign of the
// gradient's rounding noise, so the limiter must see the FP64 gradient), and
// the face pass split by a shock sensor:
//   * faces whose two cell-centre absolute pressures differ by more than the
//     factor `shock_ratio` (a captured shock or a post-shock layer's front)
//     are appended to a list and evaluated by the FP64 face kernel: the
//     reconstruction, the equation of state (rho = (p+Pref)/(R(T+Tref)),
//     material.cc:108-153) and the AUSM+up / Roe pressure terms in FP64;
//   * every other face runs in FP32 (F32: reconstruction increments formed
//     in FP64 from the FP64 gradients, then states, equation of state, flux
//     and viscous terms in float), writing its face difference as a double;
//   * the outlet faces whose right density is the reference's stale state
//     cache keep their FP64 side-stream kernel;
//   * the gather sums the face differences in FP64 in ascending face order.
// shock_ratio < 1 sends every face to FP64 (the FP64 residual);
// a huge ratio sends none.  The list order depends on the atomics, each
// face's value does not, so the result is deterministic.
#include <algorithm>

#include "ctx.hpp"

namespace fcfd {

// FP32 face pass: every face in launch order (the viscous face order of
// DevMesh::face_list, or face order) except the flagged ones, which are
// appended to `list`, and the stale-density outlet faces, which are left to
// the outlet kernel.
template <bool VISCOUS, int FX>
__global__ void __launch_bounds__(128) k_face_flux_f32(DevCase cs, DevMesh m, const double *__restrict__ W,
                                                       const double *__restrict__ G, const double *__restrict__ Lm,
                                                       double shock_ratio, double *__restrict__ D, int *__restrict__ list,
                                                       int *__restrict__ count, int *err) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  int f;
  if constexpr (VISCOUS) {
    if (i >= m.n_face_list) return;
    f = m.face_list[i];
  } else {
    if (i >= m.nf) return;
    f = i;
  }
  const int nf = m.nf;
  const int pa = m.f_parent[f], nb = m.f_neighbor[f], b = m.f_bc[f];
  const double pp = W[pa] + cs.Pref, pn = W[nb] + cs.Pref;
  const double lo = fmin(pp, pn), hi = fmax(pp, pn);
  if (shock_ratio < 1. || !(hi <= shock_ratio * lo)) {  // a pressure jump (or a non-finite pressure): FP64
    list[atomicAdd(count, 1)] = f;
    return;
  }
  const double n[3] = {m.f_n[f], m.f_n[nf + f], m.f_n[2 * nf + f]};
  const double A = m.f_area[f];
  FState<F32> L, R;
  if (!face_states<F32, 1, double>(cs, m, f, n, b, pa, nb, W, G, Lm, (F32 *)nullptr, L, R, err)) return;
  F32 Dv[5], wL;
  const GlobalGrad<double> gs{G, m.nc, pa, nb};
  face_D<F32, GlobalGrad<double>, VISCOUS, FX>(cs, m, f, n, A, b, pa, nb, L, R, gs, (const double *)nullptr, Dv, wL);
#pragma unroll
  for (int v = 0; v < 5; ++v) D[v * nf + f] = double(val(Dv[v]));
}

template <bool VISCOUS, int FX>
__device__ __forceinline__ void face_list_one(const DevCase &cs, const DevMesh &m, const double *__restrict__ W,
                                              const double *__restrict__ G, const double *__restrict__ Lm, int f,
                                              double *__restrict__ D, int *err) {
  const int nf = m.nf;
  const int pa = m.f_parent[f], nb = m.f_neighbor[f], b = m.f_bc[f];
  const double n[3] = {m.f_n[f], m.f_n[nf + f], m.f_n[2 * nf + f]};
  const double A = m.f_area[f];
  FState<double> L, R;
  if (!face_states<double, 1>(cs, m, f, n, b, pa, nb, W, G, Lm, (double *)nullptr, L, R, err)) return;
  double Dv[5], wL;
  const GlobalGrad<double> gs{G, m.nc, pa, nb};
  face_D<double, GlobalGrad<double>, VISCOUS, FX>(cs, m, f, n, A, b, pa, nb, L, R, gs, (const double *)nullptr, Dv, wL);
#pragma unroll
  for (int v = 0; v < 5; ++v) D[v * nf + f] = Dv[v];
}

// FP64 face pass over the flagged faces (count read on the device): a small
// grid striding over the list (a grid sized for every face, almost all of
// whose blocks exit at once, measured 10 us for 928 faces).
template <bool VISCOUS, int FX>
__global__ void __launch_bounds__(128) k_face_flux_list(DevCase cs, DevMesh m, const double *__restrict__ W,
                                                        const double *__restrict__ G, const double *__restrict__ Lm,
                                                        const int *__restrict__ list, const int *__restrict__ count,
                                                        double *__restrict__ D, int *err) {
  const int n = *count;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    face_list_one<VISCOUS, FX>(cs, m, W, G, Lm, list[i], D, err);
}

// The two face passes of the mixed-precision residual on x->p64 (gradients
// and limiters already formed; `count` zeroed before the launch).
void launch_mixed_faces(fcfd_ctx *x, double shock_ratio, int *list, int *count, cudaStream_t s) {
  const DevMesh &m = x->dm;
  Pipe<double> &P = x->p64;
  const int nfl = x->viscous ? m.n_face_list : m.nf;
  const int g = (nfl + 127) / 128, gl = std::min((m.nf + 127) / 128, 296);
  if (g == 0) return;
  if (x->viscous) {
    FCFD_BY_FLUX(x->cs.flux, k_face_flux_f32<true, FX><<<g, 128, 0, s>>>(x->cs, m, P.W.p, P.G.p, P.Lm.p, shock_ratio, P.D.p, list, count, x->err.p));
    FCFD_BY_FLUX(x->cs.flux, k_face_flux_list<true, FX><<<gl, 128, 0, s>>>(x->cs, m, P.W.p, P.G.p, P.Lm.p, list, count, P.D.p, x->err.p));
  } else {
    FCFD_BY_FLUX(x->cs.flux, k_face_flux_f32<false, FX><<<g, 128, 0, s>>>(x->cs, m, P.W.p, P.G.p, P.Lm.p, shock_ratio, P.D.p, list, count, x->err.p));
    FCFD_BY_FLUX(x->cs.flux, k_face_flux_list<false, FX><<<gl, 128, 0, s>>>(x->cs, m, P.W.p, P.G.p, P.Lm.p, list, count, P.D.p, x->err.p));
  }
  CK(cudaGetLastError());
}

}  // namespace fcfd
