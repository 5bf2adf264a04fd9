// A C++ caller of libfcfd_b200.so through include/fcfd.h, written the way the
// binding in INTEGRATION.md would call it from inside the reference
// (NavierStokes::b200_init / b200_residual): parse the deck, build the mesh
// from CELL-type raw arrays, create a device context, evaluate a residual, and
// report errors through status codes and fcfd_last_error().
//
// Usage: binding_check <deck> <mesh.bin> [<W.bin> <R.bin>]
//   mesh.bin: int32 n_nodes, n_cells, n_bc, conn_len, bc_len, then
//             xyz[n_nodes*3] f64, conn_index[n_cells+1], conn[conn_len],
//             bc_index[n_bc+1], bc_nodes[bc_len] (int32)
// Prints one line of key=value pairs.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <vector>

#include "fcfd.h"

template <class T>
static bool get(std::ifstream &f, T *p, size_t n) {
  f.read(reinterpret_cast<char *>(p), (std::streamsize)(n * sizeof(T)));
  return (bool)f;
}

int main(int argc, char **argv) {
  if (argc != 3 && argc != 5) {
    std::fprintf(stderr, "usage: %s <deck> <mesh.bin> [<W.bin> <R.bin>]\n", argv[0]);
    return 2;
  }
  std::printf("version=%s", fcfd_version());

  // error path: a deck that does not exist is FCFD_ERR_INPUT with a message
  fcfd_case *bad = nullptr;
  const int rc_bad = fcfd_case_from_deck("/nonexistent/deck.in", &bad);
  std::printf(" missing_deck_rc=%d missing_deck_msg_len=%zu", rc_bad, std::strlen(fcfd_last_error()));

  fcfd_case *cs = nullptr;
  int rc = fcfd_case_from_deck(argv[1], &cs);
  std::printf(" deck_rc=%d", rc);
  if (rc) { std::printf(" error=\"%s\"\n", fcfd_last_error()); return 1; }

  std::ifstream f(argv[2], std::ios::binary);
  int32_t hdr[5];
  if (!get(f, hdr, 5)) { std::printf(" mesh_file=unreadable\n"); return 1; }
  const int32_t n_nodes = hdr[0], n_cells = hdr[1], n_bc = hdr[2], conn_len = hdr[3], bc_len = hdr[4];
  std::vector<double> xyz(3 * (size_t)n_nodes);
  std::vector<int32_t> cidx(n_cells + 1), conn(conn_len), bidx(n_bc + 1), bnodes(bc_len);
  if (!get(f, xyz.data(), xyz.size()) || !get(f, cidx.data(), cidx.size()) || !get(f, conn.data(), conn.size()) ||
      !get(f, bidx.data(), bidx.size()) || !get(f, bnodes.data(), bnodes.size())) {
    std::printf(" mesh_file=short\n");
    return 1;
  }
  fcfd_raw_mesh raw{n_nodes, xyz.data(), n_cells, cidx.data(), conn.data(), n_bc, bidx.data(), bnodes.data()};
  fcfd_mesh *mesh = nullptr;
  rc = fcfd_mesh_create(&raw, cs, &mesh);
  std::printf(" mesh_rc=%d", rc);
  if (rc) { std::printf(" error=\"%s\"\n", fcfd_last_error()); return 1; }
  int64_t sz[8];
  fcfd_mesh_sizes(mesh, sz);
  std::printf(" n_cells=%lld n_faces=%lld n_ghosts=%lld", (long long)sz[0], (long long)sz[1], (long long)sz[2]);

  // reverse Cuthill-McKee order: a permutation of the cells
  {
    std::vector<int32_t> perm((size_t)sz[0]), seen((size_t)sz[0], 0);
    const int rcr = fcfd_mesh_rcm(mesh, perm.data());
    bool ok = rcr == FCFD_OK;
    for (int32_t p : perm) {
      if (p < 0 || p >= sz[0] || seen[(size_t)p]) { ok = false; break; }
      seen[(size_t)p] = 1;
    }
    std::printf(" rcm_rc=%d rcm_permutation=%d", rcr, ok ? 1 : 0);
    std::printf(" grad_weights_rc=%d", fcfd_mesh_grad_weights(mesh, nullptr));
  }

  // error path: a mesh with a cell of 7 nodes is rejected, not aborted
  std::vector<int32_t> cidx7(cidx);
  cidx7[1] = cidx7[0] + 7;
  fcfd_raw_mesh raw7 = raw;
  raw7.n_cells = 1;
  raw7.conn_index = cidx7.data();
  fcfd_mesh *m7 = nullptr;
  const int rc7 = fcfd_mesh_create(&raw7, cs, &m7);
  std::printf(" bad_mesh_rc=%d", rc7);
  if (m7) fcfd_mesh_destroy(m7);

  // error path: the context-level entry points reject a null context with a
  // status instead of dereferencing it
  {
    double z[8] = {0.};
    std::printf(" null_ctx_rc=%d,%d,%d,%d", fcfd_ctx_check(nullptr), fcfd_ctx_set_launch_overlap(nullptr, 1),
                fcfd_rans_vjp(nullptr, z, z, z, z, z, z, 0), fcfd_vjp(nullptr, z, z, z, 0));
  }

  fcfd_ctx *ctx = nullptr;
  rc = fcfd_ctx_create(mesh, cs, 0, &ctx);
  std::printf(" ctx_rc=%d", rc);
  if (rc == FCFD_OK && argc == 5) {
    std::vector<double> W(5 * (size_t)n_cells), R(5 * (size_t)n_cells);
    std::ifstream fw(argv[3], std::ios::binary);
    if (!get(fw, W.data(), W.size())) { std::printf(" state_file=short\n"); return 1; }
    rc = fcfd_residual(ctx, W.data(), R.data(), 0);
    std::printf(" residual_rc=%d", rc);
    // the mixed-precision residual with every face in FP64 equals it
    std::vector<double> R2(R.size());
    int64_t n64 = -1;
    const int rcm = fcfd_residual_mixed(ctx, W.data(), R2.data(), 0.0, 0, &n64);
    double dmax = 0., rmax = 0.;
    for (size_t i = 0; i < R.size(); ++i) {
      dmax = std::max(dmax, std::fabs(R2[i] - R[i]));
      rmax = std::max(rmax, std::fabs(R[i]));
    }
    std::printf(" mixed_rc=%d mixed_fp64_faces=%lld mixed_rel_diff=%.3e", rcm, (long long)n64, rmax > 0. ? dmax / rmax : dmax);
    std::printf(" set_kernel_bad_rc=%d", fcfd_ctx_set_gradient_kernel(ctx, 9));
    // ordinary launches give the same residual bits; no flagged error
    std::vector<double> R3(R.size());
    const int rco = fcfd_ctx_set_launch_overlap(ctx, 0);
    const int rc3 = fcfd_residual(ctx, W.data(), R3.data(), 0);
    fcfd_ctx_set_launch_overlap(ctx, 1);
    std::printf(" overlap_off_rc=%d,%d overlap_same_bits=%d check_rc=%d", rco, rc3,
                std::memcmp(R3.data(), R.data(), sizeof(double) * R.size()) == 0 ? 1 : 0, fcfd_ctx_check(ctx));
    // a laminar case has no k-omega adjoint: an input error, not a fault
    std::vector<double> K(2 * (size_t)n_cells, 1.), Wb(W.size()), Kb(K.size());
    std::printf(" rans_vjp_laminar_rc=%d",
                fcfd_rans_vjp(ctx, W.data(), K.data(), R.data(), K.data(), Wb.data(), Kb.data(), 0));
    std::ofstream fr(argv[4], std::ios::binary);
    fr.write(reinterpret_cast<const char *>(R.data()), (std::streamsize)(R.size() * sizeof(double)));
  }
  if (ctx) fcfd_ctx_destroy(ctx);
  fcfd_mesh_destroy(mesh);
  fcfd_case_destroy(cs);
  std::printf("\n");
  return 0;
}
