// Mesh builder: raw CELL-type grid -> reference-order SoA connectivity,
// geometry and least-squares stencil data for the device.
//
// The integer results (face order, parent/neighbour, boundary tags, cell face
// lists, node-neighbour lists, ghost numbering) equal those of
// Grid::create_nodes_cells / create_faces / create_boundary_ghosts
// (src/grid/grid_create_elements.cc:27-182, 184-412, 702-772) for conforming
// meshes, and every floating-point quantity is evaluated with the same
// operations in the same order as the reference (src/grid/grid.cc:123-181,
// src/set_bcs.cc:35-260, src/main.cc:456-491,
// src/face_interpolation_weights.cc:32-138, src/lsqr_grad_map.cc:32-99), with
// one rounding per operation (built with -ffp-contract=off), so the geometry is
// bit-identical.  The data structures differ: faces are discovered through a
// hash of sorted face-node tuples instead of node->cell scans, boundary node
// sets are bitmaps, and all outputs are flat arrays.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <map>
#include <unordered_map>

#include "internal.hpp"

namespace fcfd {
namespace {

struct P3 {
  double x, y, z;
};
inline P3 sub(const P3 &a, const P3 &b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline P3 add(const P3 &a, const P3 &b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline P3 scl(double s, const P3 &a) { return {s * a.x, s * a.y, s * a.z}; }
inline P3 dvd(const P3 &a, double s) { return {a.x / s, a.y / s, a.z / s}; }
inline double dot(const P3 &a, const P3 &b) { return (a.x * b.x + a.y * b.y + a.z * b.z); }
inline P3 crs(const P3 &a, const P3 &b) {
  return {a.y * b.z - a.z * b.y, -a.x * b.z + a.z * b.x, a.x * b.y - a.y * b.x};
}
inline double mag(const P3 &a) { return std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
inline P3 unit(const P3 &a) { return dvd(a, mag(a)); }

// Element face tables (CGNS node order), same faces and node order as
// grid_create_elements.cc:187-214.
const int kHexFaces[6][4] = {{0, 3, 2, 1}, {4, 5, 6, 7}, {1, 2, 6, 5}, {0, 4, 7, 3}, {1, 5, 4, 0}, {2, 3, 7, 6}};
const int kPrismFaces[5][4] = {{0, 2, 1, -1}, {3, 4, 5, -1}, {0, 3, 5, 2}, {1, 2, 5, 4}, {0, 1, 4, 3}};
const int kPyraFaces[5][4] = {{0, 3, 2, 1}, {0, 1, 4, -1}, {1, 2, 4, -1}, {3, 4, 2, -1}, {0, 4, 3, -1}};
const int kTetFaces[4][4] = {{0, 2, 1, -1}, {1, 2, 3, -1}, {0, 3, 2, -1}, {0, 1, 3, -1}};

struct FaceKey {
  std::array<int32_t, 4> n;
  bool operator==(const FaceKey &o) const { return n == o.n; }
};
struct FaceKeyHash {
  size_t operator()(const FaceKey &k) const {
    uint64_t h = 1469598103934665603ull;
    for (int v : k.n) { h ^= (uint64_t)(uint32_t)v; h *= 1099511628211ull; }
    return (size_t)h;
  }
};

bool in_box(const P3 &p, const double *c1, const double *c2) {
  const double pv[3] = {p.x, p.y, p.z};
  for (int i = 0; i < 3; ++i) {
    if (c1[i] > c2[i]) {
      if (pv[i] > c1[i] || pv[i] < c2[i]) return false;
    } else {
      if (pv[i] < c1[i] || pv[i] > c2[i]) return false;
    }
  }
  return true;
}

}  // namespace

// `faces` non-null: a face-based grid (create_faces2,
// grid_create_elements.cc:444-553), whose cell node lists in `raw` are the
// sorted node sets of the cells (grid_reader_tec.cc:236-262).
// Curvilinear gradient map of cell c (curvilinear_grad_map.cc:28-228): three
// pairs of the cell's faces define a local (xi, eta, zeta) frame; Jac row i
// is the centroid of the cell across face "plus" of pair i minus the centroid
// across face "minus"; the gradient is Jac^-T applied to the pair
// differences, i.e. weights +-Jac_invT[i] on the six cells across the faces,
// accumulated into a map keyed by cell (std::map order).
//   hexahedra: the faces (positions in the cell's face list, ascending) are
//     taken in turn, each paired with the most opposite outward normal among
//     the later faces not yet paired (first minimum of the dot product).  The
//     reference erases the current element of the std::set it is iterating
//     and then increments that iterator (lines 58-77: undefined behaviour);
//     this is the pairing that loop is written to produce.
//   other cells: every ordered choice of three face pairs over the cell's
//     faces (ascending face ids, the nested loops of lines 97-153), keeping
//     the first that maximises the determinant.
// Throws FCFD_ERR_MESH where no positive determinant exists (the reference
// would then index cell -1).
static void curvilinear_map(const fcfd_mesh &m, int c, bool hexa, const std::vector<double> &cx,
                            std::map<int32_t, P3> &gm) {
  const int j0 = m.cf_index[c], nfc = m.cf_index[c + 1] - j0;
  auto cent = [&](int k) { return P3{cx[3 * (size_t)k], cx[3 * (size_t)k + 1], cx[3 * (size_t)k + 2]}; };
  auto across = [&](int f) {
    int o = m.f_neighbor[f];
    if (o == c) o = m.f_parent[f];
    return o;
  };
  auto outward = [&](int f) {
    P3 n{m.f_normal[3 * (size_t)f], m.f_normal[3 * (size_t)f + 1], m.f_normal[3 * (size_t)f + 2]};
    if (m.f_parent[f] != c) n = scl(-1., n);
    return n;
  };
  int cp[6] = {-1, -1, -1, -1, -1, -1};
  P3 J[3] = {{0., 0., 0.}, {0., 0., 0.}, {0., 0., 0.}};
  if (hexa) {
    std::vector<int> rest;
    for (int k = 0; k < nfc; ++k) rest.push_back(k);
    int fp[6] = {-1, -1, -1, -1, -1, -1};
    int counter = 0;
    while (!rest.empty() && counter < 3) {
      const int a = rest[0];
      const P3 my = outward(m.cf_list[j0 + a]);
      double minp = 1.e20;
      int b = -1;
      for (size_t t = 1; t < rest.size(); ++t) {
        const double pr = dot(my, outward(m.cf_list[j0 + rest[t]]));
        if (pr < minp) { minp = pr; b = rest[t]; }
      }
      if (b < 0) throw Error(FCFD_ERR_MESH, "curvilinear gradient: a hexahedron face without an opposite face");
      fp[2 * counter + 1] = a;
      fp[2 * counter] = b;
      rest.erase(std::remove(rest.begin(), rest.end(), b), rest.end());
      rest.erase(rest.begin());
      ++counter;
    }
    if (counter < 3) throw Error(FCFD_ERR_MESH, "curvilinear gradient: a hexahedron without three face pairs");
    for (int i = 0; i < 3; ++i) {
      cp[2 * i + 1] = across(m.cf_list[j0 + fp[2 * i + 1]]);
      cp[2 * i] = across(m.cf_list[j0 + fp[2 * i]]);
      J[i] = sub(cent(cp[2 * i + 1]), cent(cp[2 * i]));
    }
  } else {
    std::vector<int> F(m.cf_list.begin() + j0, m.cf_list.begin() + j0 + nfc);
    std::sort(F.begin(), F.end());
    F.erase(std::unique(F.begin(), F.end()), F.end());
    const int n = (int)F.size();
    double max_det = 0.;
    bool found = false;
    int t[6];
    P3 T[3];
    for (int i1 = 0; i1 < n; ++i1)
      for (int i2 = i1; i2 < n; ++i2) {
        t[1] = across(F[i2]); t[0] = across(F[i1]);
        T[0] = sub(cent(t[1]), cent(t[0]));
        for (int i3 = i1; i3 < n; ++i3)
          for (int i4 = i3; i4 < n; ++i4) {
            t[3] = across(F[i4]); t[2] = across(F[i3]);
            T[1] = sub(cent(t[3]), cent(t[2]));
            for (int i5 = i2; i5 < n; ++i5)
              for (int i6 = i5; i6 < n; ++i6) {
                t[5] = across(F[i6]); t[4] = across(F[i5]);
                T[2] = sub(cent(t[5]), cent(t[4]));
                const double det = dot(T[0], crs(T[1], T[2]));
                if (det > max_det) {
                  max_det = det;
                  found = true;
                  for (int q = 0; q < 6; ++q) cp[q] = t[q];
                  for (int q = 0; q < 3; ++q) J[q] = T[q];
                }
              }
          }
      }
    if (!found) throw Error(FCFD_ERR_MESH, "curvilinear gradient: no face pairs with a positive determinant");
  }
  const double det = dot(J[0], crs(J[1], J[2]));
  const double a00 = J[0].x, a01 = J[0].y, a02 = J[0].z, a10 = J[1].x, a11 = J[1].y, a12 = J[1].z;
  const double a20 = J[2].x, a21 = J[2].y, a22 = J[2].z;
  P3 I[3];
  I[0].x = (a11 * a22 - a12 * a21) / det;
  I[1].x = (a02 * a21 - a01 * a22) / det;
  I[2].x = (a01 * a12 - a02 * a11) / det;
  I[0].y = (a12 * a20 - a10 * a22) / det;
  I[1].y = (a00 * a22 - a02 * a20) / det;
  I[2].y = (a02 * a10 - a00 * a12) / det;
  I[0].z = (a10 * a21 - a11 * a20) / det;
  I[1].z = (a01 * a20 - a00 * a21) / det;
  I[2].z = (a00 * a11 - a01 * a10) / det;
  gm.clear();
  gm.insert({cp[0], scl(-1., I[0])});
  for (int q = 1; q < 6; ++q) {
    const P3 &v = I[q / 2];
    const bool plus = (q & 1) != 0;
    auto it = gm.find(cp[q]);
    if (it == gm.end()) gm.insert({cp[q], plus ? v : scl(-1., v)});
    else it->second = plus ? add(it->second, v) : sub(it->second, v);
  }
}

fcfd_mesh *build_mesh(const fcfd_raw_mesh &raw, fcfd_case &cs, const FaceInput *faces) {
  auto M = new fcfd_mesh();
  fcfd_mesh &m = *M;
  try {
    const int nc = raw.n_cells;
    const int nbc = raw.n_bc;
    if ((int)cs.bc.size() != nbc)
      throw Error(FCFD_ERR_MESH, "deck has " + std::to_string(cs.bc.size()) + " BC regions, mesh has " + std::to_string(nbc));
    m.dimension = cs.dimension;
    m.nc = nc;
    // Local node ids in first-seen order over the cell connectivity.
    std::vector<int32_t> g2l(raw.n_nodes, -1);
    std::vector<int32_t> cnodes(raw.conn_index[nc]);
    int nloc = 0;
    for (int k = 0; k < raw.conn_index[nc]; ++k) {
      int gid = raw.conn[k];
      if (gid < 0 || gid >= raw.n_nodes) throw Error(FCFD_ERR_MESH, "node id out of range in connectivity");
      if (g2l[gid] < 0) {
        g2l[gid] = nloc++;
        m.nodes.push_back(raw.xyz[3 * gid]);
        m.nodes.push_back(raw.xyz[3 * gid + 1]);
        m.nodes.push_back(raw.xyz[3 * gid + 2]);
      }
      cnodes[k] = g2l[gid];
    }
    m.nnode = nloc;
    auto node = [&](int n) { return P3{m.nodes[3 * n], m.nodes[3 * n + 1], m.nodes[3 * n + 2]}; };
    // Boundary node bitmaps (local ids).
    std::vector<std::vector<uint8_t>> bcmask(nbc, std::vector<uint8_t>(nloc, 0));
    for (int b = 0; b < nbc; ++b)
      for (int k = raw.bc_index[b]; k < raw.bc_index[b + 1]; ++k) {
        int gid = raw.bc_nodes[k];
        if (gid >= 0 && gid < raw.n_nodes && g2l[gid] >= 0) bcmask[b][g2l[gid]] = 1;
      }
    // node -> interior cells, ascending (grid_create_elements.cc:114-129)
    std::vector<int32_t> nc_index(nloc + 1, 0);
    for (int c = 0; c < nc; ++c)
      for (int k = raw.conn_index[c]; k < raw.conn_index[c + 1]; ++k) nc_index[cnodes[k] + 1]++;
    for (int n = 0; n < nloc; ++n) nc_index[n + 1] += nc_index[n];
    std::vector<int32_t> nc_list(nc_index[nloc]);
    {
      std::vector<int32_t> fill(nc_index.begin(), nc_index.end() - 1);
      for (int c = 0; c < nc; ++c) {
        for (int k = raw.conn_index[c]; k < raw.conn_index[c + 1]; ++k) {
          int n = cnodes[k];
          bool dup = false;
          for (int j = nc_index[n]; j < fill[n]; ++j) if (nc_list[j] == c) dup = true;
          if (dup) throw Error(FCFD_ERR_UNSUPPORTED, "cells with repeated nodes (collapsed elements) are not supported");
          nc_list[fill[n]++] = c;
        }
      }
    }
    // Faces: key -> owner (cell, local face); created in (cell, local face)
    // order by the lower-numbered cell that carries them.
    auto ftable = [&](int nn, int cf) -> const int * {
      switch (nn) {
        case 8: return kHexFaces[cf];
        case 6: return kPrismFaces[cf];
        case 5: return kPyraFaces[cf];
        default: return kTetFaces[cf];
      }
    };
    auto nfaces_of = [&](int nn) {
      switch (nn) {
        case 8: return 6;
        case 6: return 5;
        case 5: return 5;
        case 4: return 4;
      }
      throw Error(FCFD_ERR_MESH, "unsupported element with " + std::to_string(nn) + " nodes");
    };
    std::unordered_map<FaceKey, std::pair<int32_t, int32_t>, FaceKeyHash> first;  // key -> (cell, other cell)
    first.reserve(faces ? 0 : (size_t)nc * 4);
    std::vector<int32_t> cell_nf(nc);
    // boundary face -> BC region by the region node sets (grid_create_elements.cc:318-363,
    // 498-541): the face's nodes must all be in the region; where several
    // regions match, the first one that does not also hold every node of the
    // parent cell wins; -2 (UNASSIGNED_FACE) when none matches
    auto match_bc = [&](const int *fn, int fnn, int c) {
      std::vector<int> matched;
      int cell_matched = -1;
      for (int b = 0; b < nbc; ++b) {
        bool all = true;
        for (int k = 0; k < fnn; ++k) if (!bcmask[b][fn[k]]) { all = false; break; }
        if (all) matched.push_back(b);
        if (cell_matched == -1) {
          bool callm = true;
          for (int k = raw.conn_index[c]; k < raw.conn_index[c + 1]; ++k) if (!bcmask[b][cnodes[k]]) { callm = false; break; }
          if (callm) cell_matched = b;
        }
      }
      int bcv = -2;
      if (matched.size() > 1) {
        for (int b : matched) if (b != cell_matched) { bcv = b; break; }
      } else if (matched.size() == 1) {
        bcv = matched[0];
      }
      return bcv;
    };
    m.cf_index.assign(nc + 1, 0);
    std::vector<std::vector<int32_t>> cfaces(nc);
    if (faces) {
      // file order; parent = left cell, neighbour = right cell.  The
      // reference first pads every cell's face list with one zero per face
      // (a resize meant as a reserve, grid_create_elements.cc:107-121) and
      // then appends the faces, which would add face 0 to every cell's
      // volume and stencil; the lists here hold the cell's faces only.
      for (int f = 0; f < faces->n_faces; ++f) {
        const int pa = faces->left[f], nb = faces->right[f];
        if (pa < 0 || pa >= nc) throw Error(FCFD_ERR_MESH, "face " + std::to_string(f) + " has no left cell");
        if (nb >= nc) throw Error(FCFD_ERR_MESH, "face " + std::to_string(f) + " has a right cell out of range");
        const int fnn = faces->index[f + 1] - faces->index[f];
        if (fnn < 3 || fnn > 4) throw Error(FCFD_ERR_UNSUPPORTED, "faces with " + std::to_string(fnn) + " nodes are not supported");
        int fn[4] = {-1, -1, -1, -1};
        for (int k = 0; k < fnn; ++k) {
          const int gid = faces->nodes[faces->index[f] + k];
          if (gid < 0 || gid >= raw.n_nodes || g2l[gid] < 0) throw Error(FCFD_ERR_MESH, "face node out of range");
          fn[k] = g2l[gid];
        }
        int bcv = -1;
        if (nb < 0) {
          bcv = match_bc(fn, fnn, pa);
          if (bcv < 0) throw Error(FCFD_ERR_MESH, "couldn't find BC for face " + std::to_string(f));
        }
        m.f_parent.push_back(pa);
        m.f_neighbor.push_back(nb);
        m.f_bc.push_back(bcv);
        for (int k = 0; k < 4; ++k) m.f_nodes.push_back(fn[k]);
        m.f_nn.push_back((uint8_t)fnn);
        cfaces[pa].push_back(f);
        if (nb >= 0) cfaces[nb].push_back(f);
      }
    }
    for (int c = 0; c < nc && !faces; ++c) {
      int nn = raw.conn_index[c + 1] - raw.conn_index[c];
      int nfc = nfaces_of(nn);
      cell_nf[c] = nfc;
      for (int cf = 0; cf < nfc; ++cf) {
        const int *t = ftable(nn, cf);
        FaceKey key{{-1, -1, -1, -1}};
        int fnn = (t[3] < 0) ? 3 : 4;
        for (int k = 0; k < fnn; ++k) key.n[k] = cnodes[raw.conn_index[c] + t[k]];
        std::sort(key.n.begin(), key.n.begin() + fnn);
        auto it = first.find(key);
        if (it == first.end()) first.emplace(key, std::make_pair(c, -1));
        else {
          if (it->second.second >= 0) throw Error(FCFD_ERR_MESH, "non-manifold face shared by more than two cells");
          it->second.second = c;
        }
      }
    }
    for (int c = 0; c < nc && !faces; ++c) {
      int nn = raw.conn_index[c + 1] - raw.conn_index[c];
      for (int cf = 0; cf < cell_nf[c]; ++cf) {
        const int *t = ftable(nn, cf);
        int fnn = (t[3] < 0) ? 3 : 4;
        int fn[4] = {-1, -1, -1, -1};
        for (int k = 0; k < fnn; ++k) fn[k] = cnodes[raw.conn_index[c] + t[k]];
        FaceKey key{{fn[0], fn[1], fn[2], fn[3]}};
        std::sort(key.n.begin(), key.n.begin() + fnn);
        const auto &own = first.at(key);
        if (own.first != c) continue;  // created earlier by the lower-numbered cell
        int f = (int)m.f_parent.size();
        m.f_parent.push_back(c);
        int nb = own.second;
        int bcv = -1;  // INTERNAL_FACE
        if (nb < 0) bcv = match_bc(fn, fnn, c);
        m.f_neighbor.push_back(nb);
        m.f_bc.push_back(bcv);
        for (int k = 0; k < 4; ++k) m.f_nodes.push_back(fn[k]);
        m.f_nn.push_back((uint8_t)fnn);
        cfaces[c].push_back(f);
        if (nb >= 0) cfaces[nb].push_back(f);
      }
    }
    const int nf = (int)m.f_parent.size();
    m.nf = nf;
    // Boundary regions picked by box override the grid-file tags (set_bcs.cc:50-69);
    // geometry is needed first, so the box pass runs after the face geometry.
    // ---------------- face geometry (grid.cc:123-150)
    m.f_normal.assign(3 * (size_t)nf, 0.); m.f_area.assign(nf, 0.); m.f_centroid.assign(3 * (size_t)nf, 0.);
    for (int f = 0; f < nf; ++f) {
      const int32_t *fn = &m.f_nodes[4 * (size_t)f];
      int fnn = m.f_nn[f];
      P3 nrm;
      double area;
      if (fnn == 4) {
        P3 d1 = sub(node(fn[2]), node(fn[0]));
        P3 d2 = sub(node(fn[3]), node(fn[1]));
        nrm = crs(d1, d2);
        area = 0.5 * mag(nrm);
        nrm = unit(nrm);
      } else {
        P3 av{0., 0., 0.};
        P3 c0 = node(fn[0]);
        for (int n = 1; n < fnn; ++n) {
          int nx = n + 1;
          if (nx == fnn) nx = 0;
          P3 patch = scl(0.5, crs(sub(node(fn[n]), c0), sub(node(fn[nx]), c0)));
          av = add(av, patch);
        }
        area = mag(av);
        nrm = unit(av);
      }
      P3 cen{0., 0., 0.};
      for (int n = 0; n < fnn; ++n) cen = add(cen, node(fn[n]));
      cen = dvd(cen, double(fnn));
      m.f_normal[3 * f] = nrm.x; m.f_normal[3 * f + 1] = nrm.y; m.f_normal[3 * f + 2] = nrm.z;
      m.f_area[f] = area;
      m.f_centroid[3 * f] = cen.x; m.f_centroid[3 * f + 1] = cen.y; m.f_centroid[3 * f + 2] = cen.z;
    }
    auto fnormal = [&](int f) { return P3{m.f_normal[3 * f], m.f_normal[3 * f + 1], m.f_normal[3 * f + 2]}; };
    auto fcent = [&](int f) { return P3{m.f_centroid[3 * f], m.f_centroid[3 * f + 1], m.f_centroid[3 * f + 2]}; };
    // ---------------- cell centroids and volumes (grid.cc:152-177)
    for (int c = 0; c < nc; ++c) {
      m.cf_index[c + 1] = m.cf_index[c] + (int)cfaces[c].size();
      for (int f : cfaces[c]) m.cf_list.push_back(f);
    }
    std::vector<double> cx(3 * (size_t)nc), cvol(nc);
    double total = 0.;
    for (int c = 0; c < nc; ++c) {
      P3 cen{0., 0., 0.};
      int nn = raw.conn_index[c + 1] - raw.conn_index[c];
      for (int k = raw.conn_index[c]; k < raw.conn_index[c + 1]; ++k) cen = add(cen, node(cnodes[k]));
      cen = dvd(cen, double(nn));
      double vol = 0.;
      for (int j = m.cf_index[c]; j < m.cf_index[c + 1]; ++j) {
        int f = m.cf_list[j];
        P3 ba = scl(m.f_area[f], fnormal(f));
        if (m.f_parent[f] == c) ba = scl(-1., ba);
        P3 ban = unit(ba);
        P3 h = scl(dot(sub(cen, fcent(f)), ban), ban);
        vol += dot(ba, h) / 3.;
      }
      cx[3 * c] = cen.x; cx[3 * c + 1] = cen.y; cx[3 * c + 2] = cen.z;
      cvol[c] = vol;
      total += vol;
    }
    m.total_volume = total;
    // ---------------- boundary ghosts (grid_create_elements.cc:702-741)
    std::vector<int32_t> ghost_face;
    for (int b = 0; b < nbc; ++b)
      for (int f = 0; f < nf; ++f)
        if (m.f_bc[f] == b) {
          m.f_neighbor[f] = nc + (int)ghost_face.size();
          ghost_face.push_back(f);
        }
    const int nb = (int)ghost_face.size();
    m.nb = nb;
    const int nt = nc + nb;
    m.c_centroid.assign(3 * (size_t)nt, 0.); m.c_volume.assign(nt, 0.); m.c_length.assign(nt, 0.); m.c_wall.assign(nt, 0.);
    m.c_bc.assign(nt, -1);
    std::copy(cx.begin(), cx.end(), m.c_centroid.begin());
    std::copy(cvol.begin(), cvol.end(), m.c_volume.begin());
    auto ccent = [&](int c) { return P3{m.c_centroid[3 * c], m.c_centroid[3 * c + 1], m.c_centroid[3 * c + 2]}; };
    for (int gi = 0; gi < nb; ++gi) {
      int f = ghost_face[gi], g = nc + gi, pa = m.f_parent[f];
      m.c_bc[g] = m.f_bc[f];
      m.c_volume[g] = m.c_volume[pa];
      // lengthScale is copied from the parent before set_lengthScales has run: 0
      P3 xp = ccent(pa);
      P3 gc = add(xp, scl(2. * dot(sub(fcent(f), xp), fnormal(f)), fnormal(f)));
      m.c_centroid[3 * g] = gc.x; m.c_centroid[3 * g + 1] = gc.y; m.c_centroid[3 * g + 2] = gc.z;
    }
    // Box picks run after the ghosts exist, as set_bcs runs after Grid::setup.
    // ---------------- BC region box picks (set_bcs.cc:50-69)
    for (int b = 0; b < nbc; ++b) {
      const BcRegion &R = cs.bc[b];
      if (!R.box) continue;
      for (int f = 0; f < nf; ++f) {
        if ((m.f_bc[f] >= 0 || m.f_bc[f] == -2) && in_box(fcent(f), R.corner1, R.corner2)) {
          if (R.pick == "override") m.f_bc[f] = b;
          else if (R.pick == "unassigned" && m.f_bc[f] == -2) m.f_bc[f] = b;
          else if (R.pick == "BC" && m.f_bc[f] == R.pick_from - 1) m.f_bc[f] = b;
        }
      }
    }
    for (int f = 0; f < nf; ++f)
      if (m.f_bc[f] == -2 || (m.f_bc[f] >= 0 && m.f_neighbor[f] < 0))
        throw Error(FCFD_ERR_MESH, "boundary condition could not be found for face " + std::to_string(f));
    // node -> ghost cells in creation order
    std::vector<std::vector<int32_t>> node_ghosts(nloc);
    for (int gi = 0; gi < nb; ++gi) {
      int f = ghost_face[gi];
      for (int k = 0; k < m.f_nn[f]; ++k) node_ghosts[m.f_nodes[4 * (size_t)f + k]].push_back(nc + gi);
    }
    // node neighbours (grid_create_elements.cc:131-147 then 743-769)
    m.nbr_index.assign(nc + 1, 0);
    {
      std::vector<int32_t> row;
      for (int c = 0; c < nc; ++c) {
        row.clear();
        auto push = [&](int x) {
          for (int y : row) if (y == x) return;
          row.push_back(x);
        };
        for (int k = raw.conn_index[c]; k < raw.conn_index[c + 1]; ++k) {
          int n = cnodes[k];
          for (int j = nc_index[n]; j < nc_index[n + 1]; ++j) push(nc_list[j]);
        }
        for (int k = raw.conn_index[c]; k < raw.conn_index[c + 1]; ++k)
          for (int g : node_ghosts[cnodes[k]]) push(g);
        m.nbr_list.insert(m.nbr_list.end(), row.begin(), row.end());
        m.nbr_index[c + 1] = (int)m.nbr_list.size();
      }
    }
    // ---------------- set_bcs.cc:70-93, 140-160: symmetry flags, areas, ghost centroid fix
    m.f_symmetry.assign(nf, 0);
    m.bc_total_area.assign(nbc, 0.);
    for (int b = 0; b < nbc; ++b) {
      double area = 0.;
      for (int f = 0; f < nf; ++f)
        if (m.f_bc[f] == b) {
          area += m.f_area[f];
          if (cs.bc[b].type == BC_SYMMETRY) m.f_symmetry[f] = 1;
        }
      m.bc_total_area[b] = area;
      cs.bc[b].total_area = area;
    }
    for (int f = 0; f < nf; ++f) {
      int b = m.f_bc[f];
      if (b >= 0 && (cs.bc[b].type == BC_INLET || cs.bc[b].type == BC_OUTLET)) {
        int g = m.f_neighbor[f], pa = m.f_parent[f];
        P3 xp = ccent(pa);
        P3 gc = add(xp, scl(2., sub(fcent(f), xp)));
        m.c_centroid[3 * g] = gc.x; m.c_centroid[3 * g + 1] = gc.y; m.c_centroid[3 * g + 2] = gc.z;
      }
    }
    // wall distances (set_bcs.cc:211-249): brute force over no-slip wall faces
    std::vector<int32_t> walls;
    for (int f = 0; f < nf; ++f) {
      int b = m.f_bc[f];
      if (b >= 0 && cs.bc[b].type == BC_WALL && cs.bc[b].kind != K_SLIP) walls.push_back(f);
    }
#pragma omp parallel for schedule(static)
    for (int c = 0; c < nt; ++c) {
      double best = 1.e20;
      P3 x = ccent(c);
      for (int f : walls) {
        double d = mag(sub(x, fcent(f)));
        if (best > d) best = d;
      }
      m.c_wall[c] = best;
    }
    // face wall distances and dissipation factors (set_bcs.cc:228-249), read
    // by the Steger-Warming flux only: the first closest wall face gives fN
    if (cs.flux == FLUX_SW) {
      m.f_wall.assign(nf, 1.e20);
      m.f_diss.assign(nf, 0.);
#pragma omp parallel for schedule(static)
      for (int f = 0; f < nf; ++f) {
        int b = m.f_bc[f];
        if (b < 0 || cs.bc[b].type != BC_WALL || cs.bc[b].kind == K_SLIP) {
          double best = 1.e20;
          P3 fN{0., 0., 0.}, x = fcent(f);
          for (int w : walls) {
            double d = mag(sub(x, fcent(w)));
            if (best > d) { best = d; fN = fnormal(w); }
          }
          P3 nn = fnormal(f);
          m.f_wall[f] = best;
          m.f_diss[f] = 1. - std::fabs(fN.x * nn.x + fN.y * nn.y + fN.z * nn.z);
        } else {
          m.f_wall[f] = 0.;
          m.f_diss[f] = 0.;
        }
      }
    }
    // ---------------- cell length scales (main.cc:456-489)
    for (int c = 0; c < nc; ++c) {
      double ls = 1.e20;
      for (int j = m.cf_index[c]; j < m.cf_index[c + 1]; ++j) {
        int f = m.cf_list[j];
        double h = std::fabs(dot(fnormal(f), sub(fcent(f), ccent(c))));
        bool skip = m.f_bc[f] >= 0 && cs.bc[m.f_bc[f]].type == BC_SYMMETRY;
        if (!skip) ls = std::min(ls, h);
      }
      m.c_length[c] = ls;
    }
    if (m.dimension == 3) {
      m.length_scale = std::pow(m.total_volume, 1. / 3.);
    } else {
      m.length_scale = 0.;
      for (int b = 0; b < nbc; ++b)
        if (cs.bc[b].type == BC_SYMMETRY) m.length_scale = std::max(m.length_scale, std::sqrt(0.5 * m.bc_total_area[b]));
    }
    // ---------------- tangents (ns_assemble_linear_system.cc:332-351)
    m.f_t1.assign(3 * (size_t)nf, 0.); m.f_t2.assign(3 * (size_t)nf, 0.);
    for (int f = 0; f < nf; ++f) {
      const int32_t *fn = &m.f_nodes[4 * (size_t)f];
      P3 t1;
      if (m.f_nn[f] == 4) t1 = unit(sub(add(node(fn[0]), node(fn[1])), add(node(fn[2]), node(fn[3]))));
      else t1 = unit(sub(scl(0.5, add(node(fn[0]), node(fn[1]))), fcent(f)));
      P3 t2 = unit(crs(fnormal(f), t1));
      m.f_t1[3 * f] = t1.x; m.f_t1[3 * f + 1] = t1.y; m.f_t1[3 * f + 2] = t1.z;
      m.f_t2[3 * f] = t2.x; m.f_t2[3 * f + 1] = t2.y; m.f_t2[3 * f + 2] = t2.z;
    }
    // ---------------- face averaging weights (face_interpolation_weights.cc, interpolate.cc:320-343)
    m.f_w.assign(2 * (size_t)nf, 0.);
    if (cs.interp == IP_WTLI) {
      int ms = cs.stencil_size;
      if (ms < 1) ms = (m.dimension == 3) ? 12 : (m.dimension == 2 ? 6 : 2);
      if (ms > 2) throw Error(FCFD_ERR_UNSUPPORTED, "WTLI interpolation with stencil size > 2 is not supported");
      for (int f = 0; f < nf; ++f) {
        P3 xp = ccent(m.f_parent[f]), xn = ccent(m.f_neighbor[f]);
        P3 edge = sub(xn, xp);
        P3 basis = unit(edge);
        P3 pp = sub(fcent(f), xp);
        pp = scl(dot(pp, basis), basis);
        double w1 = dot(pp, basis) / mag(edge);
        m.f_w[2 * f] = 1. - w1;
        m.f_w[2 * f + 1] = w1;
      }
    } else if (cs.interp == IP_SIMPLE) {
      for (int f = 0; f < nf; ++f) { m.f_w[2 * f] = 0.5; m.f_w[2 * f + 1] = 0.5; }
    } else {
      throw Error(FCFD_ERR_UNSUPPORTED, "IDW face interpolation is not supported on the B200 path");
    }
    // ---------------- greedy colouring of the face-neighbour graph (cells of one
    // colour share no face), used by the multicolour Gauss-Seidel preconditioner
    {
      std::vector<int32_t> col(nc, -1);
      int ncol = 0;
      std::vector<char> used;
      for (int c = 0; c < nc; ++c) {
        used.assign(ncol + 1, 0);
        for (int j = m.cf_index[c]; j < m.cf_index[c + 1]; ++j) {
          int f = m.cf_list[j];
          if (m.f_bc[f] >= 0) continue;
          int o = (m.f_parent[f] == c) ? m.f_neighbor[f] : m.f_parent[f];
          if (col[o] >= 0) used[col[o]] = 1;
        }
        int k = 0;
        while (k < ncol && used[k]) ++k;
        col[c] = k;
        if (k == ncol) ++ncol;
      }
      m.color_index.assign(ncol + 1, 0);
      for (int c = 0; c < nc; ++c) m.color_index[col[c] + 1]++;
      for (int k = 0; k < ncol; ++k) m.color_index[k + 1] += m.color_index[k];
      m.color_cells.resize(nc);
      std::vector<int32_t> fill(m.color_index.begin(), m.color_index.end() - 1);
      for (int c = 0; c < nc; ++c) m.color_cells[fill[col[c]]++] = c;
    }
    // ---------------- least-squares gradient data (lsqr_grad_map.cc:32-99)
    m.st_index.assign(nc + 1, 0);
    m.st_cof.assign(7 * (size_t)nc, 0.);
    m.st_self.assign(3 * (size_t)nc, 0.);
    m.st_recip.assign(nc, 0.);
    m.st_mirror.assign(3 * (size_t)nc, 0.);
    m.has_lsq.assign(nc, 0);
    {
      std::vector<int32_t> st;
      std::vector<P3> dist;
      std::vector<double> w;
      auto method_of = [&](int c) {
        const int nn = raw.conn_index[c + 1] - raw.conn_index[c];
        return (nn == 8) ? cs.hex_method : (nn == 6 ? cs.prism_method : cs.other_method);
      };
      // With any curvilinear cell every gradient map is stored as weights per
      // stencil entry (st_w), in the entries' key order: the device sums
      // w . phi over them instead of rebuilding least-squares weights.
      for (int c = 0; c < nc; ++c)
        if (method_of(c) == GM_CURVILINEAR) m.grad_weights = true;
      std::map<int32_t, P3> gm;
      for (int c = 0; c < nc; ++c) {
        const int nn = raw.conn_index[c + 1] - raw.conn_index[c];
        const int meth = method_of(c);
        if (meth == GM_CURVILINEAR) {
          curvilinear_map(m, c, nn == 8, m.c_centroid, gm);
          m.has_lsq[c] = 1;
          for (const auto &kv : gm) {
            m.st_keys.push_back(kv.first);
            m.st_w.push_back(kv.second.x); m.st_w.push_back(kv.second.y); m.st_w.push_back(kv.second.z);
          }
          m.st_index[c + 1] = (int)m.st_keys.size();
          continue;
        }
        if (meth == GM_GREENGAUSS) {
          // empty gradient map: the gradient falls back to Green-Gauss
          // (variable.h:204-213), evaluated per face on the device
          m.st_index[c + 1] = (int)m.st_keys.size();
          continue;
        }
        m.has_lsq[c] = 1;
        st.clear(); dist.clear(); w.clear();
        P3 xc = ccent(c);
        double a = 0., b = 0., cc = 0., d = 0., e = 0., ff = 0.;
        auto acc = [&](const P3 &dk) {
          double wk = dot(dk, dk);
          w.push_back(wk);
          dist.push_back(dk);
          a += wk * dk.x * dk.x; b += wk * dk.x * dk.y; cc += wk * dk.x * dk.z;
          d += wk * dk.y * dk.y; e += wk * dk.y * dk.z; ff += wk * dk.z * dk.z;
        };
        for (int j = m.nbr_index[c]; j < m.nbr_index[c + 1]; ++j) {
          int k = m.nbr_list[j];
          if (k == c) continue;
          st.push_back(k);
          acc(sub(ccent(k), xc));
        }
        for (int j = m.cf_index[c]; j < m.cf_index[c + 1]; ++j) {
          int f = m.cf_list[j];
          if (!m.f_symmetry[f]) continue;
          st.push_back(c);
          P3 point = add(xc, scl(dot(sub(fcent(f), xc), fnormal(f)), fnormal(f)));
          acc(sub(point, xc));
        }
        double det = a * d * ff - a * e * e - b * b * ff - cc * cc * d + 2. * b * cc * e;
        double C00 = d * ff - e * e, C01 = cc * e - b * ff, C02 = b * e - cc * d;
        double C11 = a * ff - cc * cc, C12 = b * cc - a * e, C22 = a * d - b * b;
        double *cof = &m.st_cof[7 * (size_t)c];
        cof[0] = C00; cof[1] = C01; cof[2] = C02; cof[3] = C11; cof[4] = C12; cof[5] = C22; cof[6] = det;
        // self weight: first entry inserts -w, later entries subtract (std::map semantics)
        double s0 = 0., s1 = 0., s2 = 0.;
        // Division by det through a reciprocal and one fused correction
        // (Markstein's method) is used on the device only if it reproduces the
        // IEEE quotient for every weight of this cell (checked here).
        const double recip = 1. / det;
        bool exact = std::isfinite(recip);
        double mir0 = 0., mir1 = 0., mir2 = 0.;
        for (size_t k = 0; k < st.size(); ++k) {
          const P3 &dk = dist[k];
          double w0 = w[k] * (dk.x * C00 + dk.y * C01 + dk.z * C02);
          double w1 = w[k] * (dk.x * C01 + dk.y * C11 + dk.z * C12);
          double w2 = w[k] * (dk.x * C02 + dk.y * C12 + dk.z * C22);
          for (double num : {w0, w1, w2}) {
            const double q0 = num * recip;
            const double rem = std::fma(-q0, det, num);
            const double q1 = std::fma(rem, recip, q0);
            const double qd = num / det;
            if (std::memcmp(&q1, &qd, sizeof(double)) != 0) exact = false;
          }
          w0 /= det; w1 /= det; w2 /= det;
          if (k == 0 && st[0] == c) {
            // a mirror first (no real neighbour): its insert lands and the
            // subtraction cancels it (lsqr_grad_map.cc:92-94)
            s0 = w0 - w0; s1 = w1 - w1; s2 = w2 - w2;
          } else if (k == 0) { s0 = -1. * w0; s1 = -1. * w1; s2 = -1. * w2; }
          else { s0 -= w0; s1 -= w1; s2 -= w2; }
          if (st[k] == c && k > 0) { mir0 += w0; mir1 += w1; mir2 += w2; }
        }
        m.st_recip[c] = exact ? recip : 0.;
        m.st_mirror[3 * c] = mir0; m.st_mirror[3 * c + 1] = mir1; m.st_mirror[3 * c + 2] = mir2;
        m.st_self[3 * c] = s0; m.st_self[3 * c + 1] = s1; m.st_self[3 * c + 2] = s2;
        // keys in ascending order (std::map iteration order), self included once
        std::vector<int32_t> keys(st.begin(), st.end());
        keys.push_back(c);
        std::sort(keys.begin(), keys.end());
        keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
        m.st_keys.insert(m.st_keys.end(), keys.begin(), keys.end());
        m.st_index[c + 1] = (int)m.st_keys.size();
        if (m.grad_weights) {
          // the map's weights: each neighbour's own insert (its first and
          // only occurrence), the accumulated self entry
          for (int32_t key : keys) {
            if (key == c) {
              m.st_w.push_back(s0); m.st_w.push_back(s1); m.st_w.push_back(s2);
              continue;
            }
            size_t k = 0;
            while (st[k] != key) ++k;
            const P3 &dk = dist[k];
            double w0 = w[k] * (dk.x * C00 + dk.y * C01 + dk.z * C02);
            double w1 = w[k] * (dk.x * C01 + dk.y * C11 + dk.z * C12);
            double w2 = w[k] * (dk.x * C02 + dk.y * C12 + dk.z * C22);
            w0 /= det; w1 /= det; w2 /= det;
            m.st_w.push_back(w0); m.st_w.push_back(w1); m.st_w.push_back(w2);
          }
        }
      }
    }
  } catch (...) {
    delete M;
    throw;
  }
  return M;
}

// Reverse Cuthill-McKee order of the interior cells over the face-neighbour
// graph (interior faces).  The reference orders its cells by the element
// order of the grid file and, when partitioned, by ParMETIS
// (grid_partition.cc:25-141); a grid whose elements come unordered (a
// face-based Tecplot file, a shuffled export) leaves the face kernels'
// gathers scattered over memory.  This order (Cuthill & McKee 1969, reversed
// as in George 1971) keeps face neighbours close in index, so the cells a
// warp gathers share cache lines.  Per connected component (taken in order of
// their lowest-numbered least-degree cell): a pseudo-peripheral start cell
// (Gibbs-Poole-Stockmeyer / George-Liu search: breadth-first level sets from
// the current start, move to the least-degree cell of the last level while
// the eccentricity grows), then breadth-first from it, each cell's unvisited
// neighbours in ascending (degree, index); the whole sequence is reversed.
// perm[new] = old.  Deterministic: ties always go to the lower index.
void rcm_order(const fcfd_mesh &m, std::vector<int32_t> &perm) {
  const int nc = m.nc;
  std::vector<int32_t> ai(nc + 1, 0), aj;
  for (int f = 0; f < m.nf; ++f) {
    if (m.f_bc[f] >= 0) continue;
    const int a = m.f_parent[f], b = m.f_neighbor[f];
    if (a < 0 || b < 0 || a >= nc || b >= nc || a == b) continue;
    ai[a + 1]++; ai[b + 1]++;
  }
  for (int c = 0; c < nc; ++c) ai[c + 1] += ai[c];
  aj.resize(ai[nc]);
  {
    std::vector<int32_t> fill(ai.begin(), ai.end() - 1);
    for (int f = 0; f < m.nf; ++f) {
      if (m.f_bc[f] >= 0) continue;
      const int a = m.f_parent[f], b = m.f_neighbor[f];
      if (a < 0 || b < 0 || a >= nc || b >= nc || a == b) continue;
      aj[fill[a]++] = b;
      aj[fill[b]++] = a;
    }
  }
  // distinct neighbours (two cells can share more than one face), then
  // ascending (degree, index)
  std::vector<int32_t> deg(nc);
  {
    std::vector<int32_t> ai2(nc + 1, 0), aj2;
    aj2.reserve(aj.size());
    for (int c = 0; c < nc; ++c) {
      std::vector<int32_t> v(aj.begin() + ai[c], aj.begin() + ai[c + 1]);
      std::sort(v.begin(), v.end());
      v.erase(std::unique(v.begin(), v.end()), v.end());
      aj2.insert(aj2.end(), v.begin(), v.end());
      ai2[c + 1] = (int32_t)aj2.size();
    }
    ai.swap(ai2);
    aj.swap(aj2);
    for (int c = 0; c < nc; ++c) deg[c] = ai[c + 1] - ai[c];
    for (int c = 0; c < nc; ++c)
      std::sort(aj.begin() + ai[c], aj.begin() + ai[c + 1],
                [&](int32_t a, int32_t b) { return deg[a] != deg[b] ? deg[a] < deg[b] : a < b; });
  }
  std::vector<uint8_t> done(nc, 0);
  std::vector<int32_t> level(nc, -1), order;
  order.reserve(nc);
  // breadth-first level sets from r over the not-yet-ordered cells; returns
  // the eccentricity and the least-degree (lowest index) cell of the last level
  std::vector<int32_t> touched;
  auto bfs_last = [&](int r, int &ecc) -> int {
    touched.clear();
    std::vector<int32_t> cur{r}, nxt;
    level[r] = 0;
    touched.push_back(r);
    ecc = 0;
    std::vector<int32_t> last = cur;
    while (!cur.empty()) {
      nxt.clear();
      for (int c : cur)
        for (int k = ai[c]; k < ai[c + 1]; ++k) {
          const int o = aj[k];
          if (done[o] || level[o] >= 0) continue;
          level[o] = level[c] + 1;
          touched.push_back(o);
          nxt.push_back(o);
        }
      if (nxt.empty()) break;
      ++ecc;
      last = nxt;
      cur.swap(nxt);
    }
    for (int c : touched) level[c] = -1;
    int best = last[0];
    for (int c : last)
      if (deg[c] < deg[best] || (deg[c] == deg[best] && c < best)) best = c;
    return best;
  };
  for (;;) {
    int seed = -1;
    for (int c = 0; c < nc; ++c)
      if (!done[c] && (seed < 0 || deg[c] < deg[seed])) seed = c;
    if (seed < 0) break;
    int ecc = 0;
    int cand = bfs_last(seed, ecc);
    for (;;) {
      int ecc2 = 0;
      const int cand2 = bfs_last(cand, ecc2);
      if (ecc2 <= ecc) break;
      seed = cand;
      ecc = ecc2;
      cand = cand2;
    }
    // Cuthill-McKee from the pseudo-peripheral cell `seed`
    size_t head = order.size();
    order.push_back(seed);
    done[seed] = 1;
    while (head < order.size()) {
      const int c = order[head++];
      for (int k = ai[c]; k < ai[c + 1]; ++k) {
        const int o = aj[k];
        if (done[o]) continue;
        done[o] = 1;
        order.push_back(o);
      }
    }
  }
  perm.assign(order.rbegin(), order.rend());
}

}  // namespace fcfd
