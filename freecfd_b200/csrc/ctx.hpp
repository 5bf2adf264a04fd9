// Device context shared by the residual (fcfd.cu) and the Newton-Krylov
// solver (newton.cu).
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <type_traits>
#include <vector>

#include "internal.hpp"
#include "kernels.cuh"

namespace fcfd {

#define CK(call)                                                                                        \
  do {                                                                                                  \
    cudaError_t e_ = (call);                                                                            \
    if (e_ != cudaSuccess) throw Error(FCFD_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

template <class T>
struct DBuf {
  T *p = nullptr;
  size_t n = 0;
  void alloc(size_t count) {
    free();
    n = count;
    if (count) CK(cudaMalloc(&p, count * sizeof(T)));
  }
  void upload(const std::vector<T> &v) {
    alloc(v.size());
    if (n) CK(cudaMemcpy(p, v.data(), n * sizeof(T), cudaMemcpyHostToDevice));
  }
  void free() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  ~DBuf() { free(); }
};

// [n][k] AoS host array -> [k][n] SoA
template <class T>
static std::vector<T> soa(const std::vector<T> &a, size_t n, int k) {
  std::vector<T> o(a.size());
  for (size_t i = 0; i < n; ++i)
    for (int j = 0; j < k; ++j) o[j * n + i] = a[i * k + j];
  return o;
}

struct Timing {
  cudaEvent_t ev[8];
  Timing() { for (auto &e : ev) cudaEventCreate(&e); }
  ~Timing() { for (auto &e : ev) cudaEventDestroy(e); }
};

}  // namespace fcfd


namespace fcfd {
// Typed working buffers of one residual chain (scalar S = double, or a dual
// number for tangent runs).
template <class S>
struct Pipe {
  DBuf<S> W, G, Lm, D, stale, R;
  bool ready = false;
  void alloc(int nc, int nf, int nb) {
    const int nt = nc + nb;
    W.alloc(5 * (size_t)nt); G.alloc(15 * (size_t)nc); Lm.alloc(5 * (size_t)nc); D.alloc(5 * (size_t)nf);
    stale.alloc(nb > 0 ? nb : 1); R.alloc(5 * (size_t)nc);
    CK(cudaMemset(stale.p, 0, sizeof(S) * (nb > 0 ? nb : 1)));
    ready = true;
  }
};
}  // namespace fcfd

namespace fcfd {
struct AdjointState;  // adjoint.cu: buffers of the reverse sweep, allocated on first use
struct RansState;     // rans.cu: k-omega state and buffers (turbulent cases)
}

using namespace fcfd;  // internal header: the context mirrors the device types

struct fcfd_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  // outlet-face fluxes run on `side`, forked from and joined back to `stream`
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  DevCase cs{};
  DevMesh dm{};
  const fcfd_mesh *mesh = nullptr;
  const fcfd_case *case_ptr = nullptr;
  bool viscous = false;
  // mesh arrays
  DBuf<int> f_parent, f_neighbor, f_bc, cf_index, cf_list, st_index, st_keys, bface, outlet, color_cells;
  std::vector<int> color_index;
  // Gauss-Seidel couplings packed per colour, slot-major [gs_deg][cells of the
  // colour]: the neighbour across each interior face and the signed face
  DBuf<int> gs_nbr, gs_src;
  int gs_deg = 0;
  DBuf<double> f_n, f_area, f_x, f_w, c_x, c_len, st_cof, st_self, st_recip, st_mirror, c_vol, f_wall, f_diss;
  DBuf<double> st_w;  // stored gradient-map weights [E][3] (curvilinear cases)
  bool green_gauss = false;  // some cells take the Green-Gauss gradient
  // state arrays
  Pipe<double> p64;
  Pipe<Dual<double>> pjv;
  Pipe<Dual<float>> pjv32;  // FP32 tangent chain (mixed-precision Newton-Krylov)
  DBuf<double> Win, Vin, Rtmp, dt, mdot, wl;
  AdjointState *adj = nullptr;
  RansState *rans = nullptr;
  DBuf<unsigned long long> ext;    // global extrema slots of the VK limiter (armed between chains)
  DBuf<unsigned long long> dtmin;  // CFL_MAX minimum of the local time step
  DBuf<int> err, argx;
  DBuf<unsigned char> flush;
  int n_outlet = 0;
  cudaGraphExec_t graph = nullptr;  // the timed residual chain
  int graph_fast_grad = -1;
  // fcfd_residual with pinned host buffers: copy in, chain, copy out and the
  // error flag as one graph, kept for the last (W, R) pair
  cudaGraphExec_t host_graph = nullptr;
  const double *host_graph_W = nullptr;
  double *host_graph_R = nullptr;
  int host_graph_fast_grad = -1;
  int *err_pinned = nullptr;
  bool newton_frozen = false;
  bool newton_f32 = false;  // Krylov matvecs through the FP32 tangent chain
  // one rank's part of a domain-decomposed residual: `dm` with the partition
  // lists set (the PART instantiations of the chain's kernels use it)
  DevMesh dmp{};
  DBuf<int> part_cells, part_faces, part_outlet, part_ghosts;
  DBuf<int> face_order;  // faces grouped by kind (DevMesh::face_list of the whole mesh)
  // mixed-precision residual: faces sent to the FP64 pass, and their count
  DBuf<int> mx_list, mx_count;
  // tiles of the shared-memory gradient kernel (DevMesh::tile_off ...)
  DBuf<int> tile_off, tile_cells, st_local, cf_local, self_local;
  // folded stencils of the fused gradient (DevMesh::fold_index ...)
  DBuf<int> fold_index, fold_key;
  DBuf<double> fold_e;
  int grad_kernel = 0;  // fcfd_ctx_set_gradient_kernel: 0 automatic, 1 per cell, 2 tiles
  // the residual chain's gradient and face launches overlap their
  // predecessor's tail (programmatic dependent launch); fcfd_ctx_set_launch_overlap
  bool pdl = true;
};


namespace fcfd {
constexpr int kExtremaBlocks = 296;  // 2 x 148 SMs

// Launches kernel k; with pdl, as a programmatic dependent launch (it may be
// scheduled before its stream predecessor completes and waits for it in
// pdl_wait()).
template <class... KP, class... A>
inline void launch_k(bool pdl, void (*k)(KP...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, A... args) {
  if (!pdl) {
    k<<<grid, block, smem, s>>>(args...);
    return;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  CK(cudaLaunchKernelEx(&cfg, k, args...));
}
constexpr int kPairGradCells = 148 * 512;
template <class S>
void launch_chain(fcfd_ctx *x, Pipe<S> &P, S *Rout, bool aos_out, S *mo, S *wo, bool frozen_limiter = false);
int check_err(fcfd_ctx *x);

// Gradient + limiter launch: the fused-gradient and bit-exact instantiations
// are separate kernels so each gets the registers its own path needs.
// PART: the gradient cells of one rank of a domain decomposition (m = dmp).
template <class S, bool PART = false>
inline void launch_grad_limiter(const DevCase &cs, const DevMesh &m, const S *W, const unsigned long long *ext,
                                const int *argx, S *G, S *Lm, cudaStream_t s, bool pdl = false) {
  const int g = ((PART ? m.n_part_cells : m.nc) + 127) / 128;
  if (g == 0) return;
  if constexpr (std::is_same<S, double>::value && !PART) {
    if (cs.tile_grad && m.tile_off) {
      const int nt_ = (m.nc + kGradTile - 1) / kGradTile;
      const size_t smem = sizeof(double) * 8 * (size_t)m.tile_slots_max;
      if (cs.fast_grad) launch_k(pdl, k_grad_limiter_tile<true>, nt_, kGradTile, smem, s, cs, m, W, ext, G, Lm);
      else launch_k(pdl, k_grad_limiter_tile<false>, nt_, kGradTile, smem, s, cs, m, W, ext, G, Lm);
      return;
    }
  }
  if constexpr (std::is_same<S, double>::value) {
    // meshes too small to fill the GPU with one thread per cell (fewer than
    // 148 SMs x 512 cells) take two threads per cell
    const int ncell = PART ? m.n_part_cells : m.nc;
    if (cs.fast_grad && cs.pair_grad && ncell < kPairGradCells) {
      launch_k(pdl, k_grad_limiter_pair<PART>, (ncell + 31) / 32, 64, 0, s, cs, m, W, ext, G, Lm);
      return;
    }
  }
  if (cs.fast_grad)
    launch_k(pdl, k_grad_limiter<S, true, PART>, g, 128, 0, s, cs, m, W, ext, argx, G, Lm);
  else
    launch_k(pdl, k_grad_limiter<S, false, PART>, g, 128, 0, s, cs, m, W, ext, argx, G, Lm);
}
// Face fluxes of one residual: the main launch over all faces and, when the
// mesh has outlet faces, the outlet-face launch (stale right densities) on the
// side stream, forked after the gradient kernel and joined before the gather.
// PART: the faces of one rank of a domain decomposition (x->dmp).
template <class S, bool PART = false>
inline void launch_faces(fcfd_ctx *x, Pipe<S> &P, const S *mu_t, S *mo, S *wo, cudaStream_t s) {
  const DevMesh &m = PART ? x->dmp : x->dm;
  const int no = PART ? m.n_part_outlet : m.n_outlet, nfl = (PART || x->viscous) ? m.n_face_list : m.nf;
  const bool side = no > 0;
  if (side) {
    CK(cudaEventRecord(x->ev_fork, s));
    CK(cudaStreamWaitEvent(x->side, x->ev_fork, 0));
    const int g = (no + 127) / 128;
    if (x->viscous)
      FCFD_BY_FLUX(x->cs.flux, k_face_flux<S, true, FX, true, PART><<<g, 128, 0, x->side>>>(x->cs, m, P.W.p, P.G.p, P.Lm.p, P.stale.p, mu_t, P.D.p, mo, wo, x->err.p));
    else
      FCFD_BY_FLUX(x->cs.flux, k_face_flux<S, false, FX, true, PART><<<g, 128, 0, x->side>>>(x->cs, m, P.W.p, P.G.p, P.Lm.p, P.stale.p, mu_t, P.D.p, mo, wo, x->err.p));
    CK(cudaEventRecord(x->ev_join, x->side));
  }
  const int g = (nfl + 127) / 128;
  const bool pdl = x->pdl;
  if (g > 0 && x->viscous)
    FCFD_BY_FLUX(x->cs.flux, launch_k(pdl, k_face_flux<S, true, FX, false, PART>, g, 128, 0, s, x->cs, m, P.W.p, P.G.p, P.Lm.p, P.stale.p, mu_t, P.D.p, mo, wo, x->err.p));
  else if (g > 0)
    FCFD_BY_FLUX(x->cs.flux, launch_k(pdl, k_face_flux<S, false, FX, false, PART>, g, 128, 0, s, x->cs, m, P.W.p, P.G.p, P.Lm.p, P.stale.p, mu_t, P.D.p, mo, wo, x->err.p));
  if (side) CK(cudaStreamWaitEvent(s, x->ev_join, 0));
}
// newton.cu: inverse flow-equation blocks of the block-Jacobi preconditioner
// at the state of the last residual chain (see there).
void ns_block_inverse(fcfd_ctx *x, const double *Wn, const double *vol, const double *dt, const double *mutf,
                      double *JL, double *JR, double *Minv, double *rowmag);
void adjoint_free(fcfd_ctx *x);
// rans.cu: the coupled implicit step of the time-marching driver for turbulent
// decks (an opaque driver state: X = (W, K), its residual, the Krylov solve)
void *kw_driver_create(fcfd_ctx *x, const double *W, const double *K, int mdim);
void kw_driver_destroy(void *p);
void kw_driver_residual(fcfd_ctx *x, void *p);
int kw_driver_step(fcfd_ctx *x, void *p, const double *dt, int mode, double krtol, double kabstol);
void kw_driver_update(fcfd_ctx *x, void *p, const double *dt, double *part, int *err);
void kw_driver_state(fcfd_ctx *x, void *p, double *W, double *K, double *mut);

// The coupled NS + k-omega evaluation at (W, K) (device AoS [nc][5], [nc][2])
// that the adjoint reverses: leaves W with its ghosts in x->p64.W and these
// device arrays (SoA) of the same evaluation.
struct RansFwd {
  const double *K;     // [2][nt] k, omega with the ghosts' values
  const double *GK;    // [6][nc] k, omega gradients
  const double *mut;   // [nt] eddy viscosity
  const double *mutf;  // [nf] its face values
  const double *mdot;  // [nf] NS face mass flux
  const double *wl;    // [nf] NS face left weight
  const double *vol;   // [nc] cell volumes
  double ratio;        // eddy viscosity ratio limit
};
void rans_eval_for_adjoint(fcfd_ctx *x, const double *W, const double *K, RansFwd &out);
// mixed.cu: FP32 face pass + FP64 pass over the shock-flagged faces
void launch_mixed_faces(fcfd_ctx *x, double shock_ratio, int *list, int *count, cudaStream_t s);
void rans_setup(fcfd_ctx *x);
void rans_free(fcfd_ctx *x);
}  // namespace fcfd
