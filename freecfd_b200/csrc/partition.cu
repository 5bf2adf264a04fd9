// One rank's part of a domain-decomposed residual.
//
// The reference partitions the grid with ParMETIS (grid_partition.cc), keeps
// one layer of partition ghosts per rank, exchanges their primitives
// (NavierStokes::mpi_update_ghost_primitives, ns_mpi.cc:62-140) and gradients
// (mpi_update_ghost_gradients) every residual, and all-reduces the limiter's
// extrema (find_min_max, ns.cc:425-427).  Here a rank owns the contiguous
// global cell range [lo, hi) and keeps the whole mesh resident (connectivity
// and geometry are set-up data; the device holds them once per rank), but
// evaluates only its own part of each kernel:
//   * fluxes of every face of an owned cell;
//   * gradient and limiter of every cell those faces reconstruct from: the
//     owned cells, their face neighbours, and the cells the stale outlet
//     density walks back to (the state cache of ns_state_cache.h, read at
//     outlet faces, comes from the previous face in face order);
//   * ghosts of every boundary face whose parent's state is current.
// The states needed are those cells plus their LSQ stencils (node neighbours)
// and the two cells the VK extrema quirk reads (T of cell 0, w of the last
// cell): the halo, received from the ranks owning it, so the state is
// exchanged once per residual and gradients are recomputed on the halo rather
// than exchanged.  The owned rows of R equal the single-domain residual bit
// for bit, because every cell and face quantity is formed by the same
// arithmetic from the same inputs.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "ctx.hpp"

namespace fcfd {

extern template __global__ void k_ghost_minmax<double>(DevCase, DevMesh, double *, unsigned long long *, int *);
void set_last_error(const std::string &m);

namespace {

struct PartSets {
  std::vector<int> grad, faces, outlet_idx, ghosts, halo;
};

PartSets partition_sets(const fcfd_mesh &m, const fcfd_case &c, int lo, int hi) {
  const int nc = m.nc, nf = m.nf, nb = m.nb;
  if (lo < 0 || hi > nc || lo >= hi) throw Error(FCFD_ERR_INPUT, "partition range must satisfy 0 <= lo < hi <= cells");
  std::vector<char> inF(nf, 0), inE(nc, 0), cur(nc, 0);
  std::vector<int> bface(nb, -1);
  for (int f = 0; f < nf; ++f)
    if (m.f_bc[f] >= 0) bface[m.f_neighbor[f] - nc] = f;
  for (int cc = lo; cc < hi; ++cc) {
    inE[cc] = 1;
    for (int j = m.cf_index[cc]; j < m.cf_index[cc + 1]; ++j) inF[m.cf_list[j]] = 1;
  }
  for (int f = 0; f < nf; ++f) {
    if (!inF[f]) continue;
    if (m.f_bc[f] < 0) {
      inE[m.f_parent[f]] = 1;
      inE[m.f_neighbor[f]] = 1;
    } else if (c.bc[m.f_bc[f]].type == BC_OUTLET) {
      // the stale right density: walk back to the first interior face (every
      // face it may stop at contributes its reconstructing cell)
      for (int g = f - 1; g >= 0; --g) {
        if (m.f_bc[g] < 0) { inE[m.f_neighbor[g]] = 1; break; }
        inE[m.f_parent[g]] = 1;
      }
    }
  }
  for (int cc = 0; cc < nc; ++cc) {
    if (!inE[cc]) continue;
    cur[cc] = 1;
    for (int j = m.st_index[cc]; j < m.st_index[cc + 1]; ++j) {
      const int k = m.st_keys[j];
      if (k < nc) cur[k] = 1;
      else cur[m.f_parent[bface[k - nc]]] = 1;
    }
    for (int j = m.cf_index[cc]; j < m.cf_index[cc + 1]; ++j) {
      const int f = m.cf_list[j];
      if (m.f_bc[f] < 0) cur[m.f_parent[f] == cc ? m.f_neighbor[f] : m.f_parent[f]] = 1;
    }
  }
  cur[0] = 1;
  cur[nc - 1] = 1;
  PartSets P;
  for (int cc = 0; cc < nc; ++cc) {
    if (inE[cc]) P.grad.push_back(cc);
    if (cur[cc] && (cc < lo || cc >= hi)) P.halo.push_back(cc);
  }
  int oi = 0;
  for (int f = 0; f < nf; ++f) {
    const bool outlet = m.f_bc[f] >= 0 && c.bc[m.f_bc[f]].type == BC_OUTLET;
    if (inF[f]) {
      P.faces.push_back(f);
      if (outlet) P.outlet_idx.push_back(oi);
    }
    if (outlet) ++oi;
  }
  for (int t = 0; t < nb; ++t)
    if (cur[m.f_parent[bface[t]]]) P.ghosts.push_back(t);
  // faces grouped by kind like the whole mesh's face list (interior, then
  // each BC region), face order within a group
  std::stable_sort(P.faces.begin(), P.faces.end(), [&](int a, int b) { return m.f_bc[a] < m.f_bc[b]; });
  return P;
}

// ordered keys of the extrema slots, host side (the device's okey/okey_inv)
unsigned long long host_okey(double x) {
  unsigned long long b;
  std::memcpy(&b, &x, 8);
  return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
double host_okey_inv(unsigned long long k) {
  const unsigned long long b = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
  double x;
  std::memcpy(&x, &b, 8);
  return x;
}

// extrema slots: arm (even: max, key 0; odd: min, all ones), read out as
// doubles (+-inf where no cell reached the slot), set from doubles
__global__ void k_ext_arm(unsigned long long *key) {
  const int t = threadIdx.x;
  if (t < 8) key[t] = (t & 1) ? ~0ull : 0ull;
}
__global__ void k_ext_out(const unsigned long long *__restrict__ key, double *__restrict__ ext) {
  const int t = threadIdx.x;
  if (t >= 8) return;
  const unsigned long long k = key[t], armed = (t & 1) ? ~0ull : 0ull;
  ext[t] = (k == armed) ? ((t & 1) ? INFINITY : -INFINITY) : okey_inv(k);
}
__global__ void k_ext_in(const double *__restrict__ ext, unsigned long long *__restrict__ key) {
  const int t = threadIdx.x;
  if (t < 8) key[t] = okey(ext[t]);
}

template <class F>
int api(F &&body) {
  try {
    body();
  } catch (const Error &e) {
    set_last_error(e.what());
    return e.code;
  } catch (const std::exception &e) {
    set_last_error(e.what());
    return FCFD_ERR_INPUT;
  }
  return FCFD_OK;
}

}  // namespace
}  // namespace fcfd

using namespace fcfd;

extern "C" int fcfd_partition_sets(const fcfd_mesh *mesh, const fcfd_case *cs, int lo, int hi, int counts[4],
                                   int *grad_cells, int *faces, int *halo) {
  return api([&] {
    if (!mesh || !cs || !counts) throw Error(FCFD_ERR_INPUT, "null argument");
    const PartSets P = partition_sets(*mesh, *cs, lo, hi);
    counts[0] = (int)P.grad.size();
    counts[1] = (int)P.faces.size();
    counts[2] = (int)P.halo.size();
    counts[3] = (int)P.ghosts.size();
    if (grad_cells) std::copy(P.grad.begin(), P.grad.end(), grad_cells);
    if (faces) std::copy(P.faces.begin(), P.faces.end(), faces);
    if (halo) std::copy(P.halo.begin(), P.halo.end(), halo);
  });
}

extern "C" int fcfd_ctx_set_partition(fcfd_ctx *x, int lo, int hi) {
  return api([&] {
    if (!x) throw Error(FCFD_ERR_INPUT, "null argument");
    CK(cudaSetDevice(x->device));
    if (lo == 0 && hi == 0) {
      x->dmp = DevMesh{};
      return;
    }
    if (x->case_ptr->turbulent)
      throw Error(FCFD_ERR_UNSUPPORTED, "the partitioned residual covers laminar and Euler cases (no k-omega terms)");
    const PartSets P = partition_sets(*x->mesh, *x->case_ptr, lo, hi);
    x->part_cells.upload(P.grad);
    x->part_faces.upload(P.faces);
    x->part_outlet.upload(P.outlet_idx.empty() ? std::vector<int>{0} : P.outlet_idx);
    x->part_ghosts.upload(P.ghosts.empty() ? std::vector<int>{0} : P.ghosts);
    DevMesh d = x->dm;
    d.part_cells = x->part_cells.p; d.n_part_cells = (int)P.grad.size();
    d.face_list = x->part_faces.p; d.n_face_list = (int)P.faces.size();
    d.part_outlet = x->part_outlet.p; d.n_part_outlet = (int)P.outlet_idx.size();
    d.part_ghosts = x->part_ghosts.p; d.n_part_ghosts = (int)P.ghosts.size();
    d.own_lo = lo; d.own_hi = hi;
    x->dmp = d;
    CK(cudaStreamSynchronize(x->stream));
  });
}

// The stream a context's work runs on, for callers that enqueue their own
// work around it (a halo exchange, the extrema all-reduce).
extern "C" int fcfd_ctx_check(fcfd_ctx *x) {
  return api([&] {
    if (!x) throw Error(FCFD_ERR_INPUT, "null context");
    CK(cudaSetDevice(x->device));
    check_err(x);
  });
}

extern "C" int fcfd_ctx_stream(const fcfd_ctx *x, void **stream) {
  return api([&] {
    if (!x || !stream) throw Error(FCFD_ERR_INPUT, "null argument");
    *stream = (void *)x->stream;
  });
}

// Phase 1 of a partitioned residual: load W (all rows; only owned and halo
// rows need be current), update the partition's ghosts and reduce the VK
// extrema over the owned cells.  ext[0..8): max p, min p, max u, min u,
// max v, min v, max p and min p over cells below the last one (+-inf where
// the owned range has no such cell); combine across ranks with max (even
// slots) and min (odd slots).  With FCFD_DEVICE_PTRS, W and ext are device
// pointers and the call only enqueues work on the context's stream (BC
// errors are reported by phase 2).
extern "C" int fcfd_partition_extrema(fcfd_ctx *x, const double *W, double ext[8], int flags) {
  return api([&] {
    if (!x || !W || !ext) throw Error(FCFD_ERR_INPUT, "null argument");
    if (!x->dmp.part_cells) throw Error(FCFD_ERR_INPUT, "no partition set (fcfd_ctx_set_partition)");
    CK(cudaSetDevice(x->device));
    const DevMesh &m = x->dmp;
    cudaStream_t s = x->stream;
    const double *win = W;
    if (!(flags & FCFD_DEVICE_PTRS)) {
      CK(cudaMemcpyAsync(x->Win.p, W, sizeof(double) * 5 * m.nc, cudaMemcpyHostToDevice, s));
      win = x->Win.p;
    }
    k_aos_to_soa<double><<<(m.nc + 255) / 256, 256, 0, s>>>(win, x->p64.W.p, m.nc, m.nt);
    k_ext_arm<<<1, 32, 0, s>>>(x->ext.p);
    const bool need_ext = x->cs.limiter == 1 && x->cs.order != 1;
    const int tb = 256;
    const int ng = (n_ghost_threads(m) + tb - 1) / tb + (need_ext ? kExtremaBlocks : 0);
    if (ng > 0) k_ghost_minmax<double><<<ng, tb, 0, s>>>(x->cs, m, x->p64.W.p, need_ext ? x->ext.p : nullptr, x->err.p);
    if (flags & FCFD_DEVICE_PTRS) {
      k_ext_out<<<1, 32, 0, s>>>(x->ext.p, ext);
      CK(cudaGetLastError());
      return;
    }
    const unsigned long long armed[8] = {0ull, ~0ull, 0ull, ~0ull, 0ull, ~0ull, 0ull, ~0ull};
    unsigned long long k[8];
    CK(cudaMemcpyAsync(k, x->ext.p, sizeof(k), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    for (int i = 0; i < 8; ++i) ext[i] = (k[i] == armed[i]) ? ((i & 1) ? INFINITY : -INFINITY) : host_okey_inv(k[i]);
    check_err(x);
  });
}

// Phase 2: with the extrema combined over all ranks, gradient + limiter,
// face fluxes and the gather of the owned rows (R [nc][5]; only rows
// [lo, hi) are written).  Uses the state and ghosts of the last phase 1.
// With FCFD_DEVICE_PTRS, ext and R are device pointers.
extern "C" int fcfd_partition_residual(fcfd_ctx *x, const double ext[8], double *R, int flags) {
  return api([&] {
    if (!x || !ext || !R) throw Error(FCFD_ERR_INPUT, "null argument");
    if (!x->dmp.part_cells) throw Error(FCFD_ERR_INPUT, "no partition set (fcfd_ctx_set_partition)");
    CK(cudaSetDevice(x->device));
    const DevMesh &m = x->dmp;
    cudaStream_t s = x->stream;
    const bool dev = flags & FCFD_DEVICE_PTRS;
    if (dev) {
      k_ext_in<<<1, 32, 0, s>>>(ext, x->ext.p);
    } else {
      unsigned long long k[8];
      for (int i = 0; i < 8; ++i) k[i] = host_okey(ext[i]);
      CK(cudaMemcpyAsync(x->ext.p, k, sizeof(k), cudaMemcpyHostToDevice, s));
    }
    Pipe<double> &P = x->p64;
    launch_grad_limiter<double, true>(x->cs, m, P.W.p, x->ext.p, nullptr, P.G.p, P.Lm.p, s);
    launch_faces<double, true>(x, P, (const double *)nullptr, x->mdot.p, x->wl.p, s);
    double *rout = dev ? R : x->Rtmp.p;
    const int tb = 256;
    k_gather<double, true><<<(5 * n_owned(m) + tb - 1) / tb, tb, 0, s>>>(m, P.D.p, rout, x->ext.p, x->argx.p);
    CK(cudaGetLastError());
    if (!dev)
      CK(cudaMemcpyAsync(R + 5 * (size_t)m.own_lo, x->Rtmp.p + 5 * (size_t)m.own_lo,
                         sizeof(double) * 5 * (size_t)n_owned(m), cudaMemcpyDeviceToHost, s));
    // enqueue only: the error flag stays on the device for fcfd_ctx_check
    if (dev && (flags & FCFD_NO_SYNC)) return;
    CK(cudaStreamSynchronize(s));
    check_err(x);
  });
}
