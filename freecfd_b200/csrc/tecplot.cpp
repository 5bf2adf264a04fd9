// Tecplot FEPolyhedron grid reader (Grid::readTEC, src/grid/grid_reader_tec.cc:36-278).
//
// File layout the reference reads: header lines up to the first line whose
// first non-blank character is a digit or '-', each split at ',' into
// `key=value` expressions (Nodes, Elements, Faces, ZONETYPE=FEPolyhedron,
// DATAPACKING=BLOCK, NumConnectedBoundaryFaces=0, TotalNumBoundaryConnections
// =0); then, with at most one comment line before each block, the x, y and z
// node coordinates, the node count of every face, the face node lists
// (1-based), the left and the right element of every face (1-based, 0 = no
// element).  Boundary zones follow, one per BC region in BC order: header lines
// with `ZONE T="name"` and `Nodes=n`, then the x, y, z coordinates of the
// zone's nodes; each is matched to the nearest node of a boundary face (the
// reference uses a kd-tree; here an exact coordinate lookup, else the nearest
// by brute force, the lowest node id among equals); the rest of the zone up to
// the next line starting with ZONE is skipped.  A cell's node list is the
// sorted set of its faces' nodes (grid_reader_tec.cc:236-262).
#include <algorithm>
#include <array>
#include <cctype>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <set>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>

#include "internal.hpp"

namespace fcfd {

fcfd_mesh *build_mesh(const fcfd_raw_mesh &raw, fcfd_case &cs, const FaceInput *faces);

namespace {

// A cursor over the file text with the stream operations readTEC uses.
struct Cursor {
  std::string t;
  size_t p = 0;
  bool eof() const { return p >= t.size(); }
  // is_first_numeric: skip blanks, then is the next character a digit or '-'?
  bool first_numeric() {
    while (p < t.size() && std::isspace((unsigned char)t[p])) ++p;
    return p < t.size() && (t[p] == '-' || std::isdigit((unsigned char)t[p]));
  }
  bool getline(std::string &line) {
    if (p >= t.size()) { line.clear(); return false; }
    size_t e = t.find('\n', p);
    if (e == std::string::npos) e = t.size();
    line = t.substr(p, e - p);
    p = (e < t.size()) ? e + 1 : e;
    return true;
  }
  template <class T>
  T number(const char *what) {
    while (p < t.size() && std::isspace((unsigned char)t[p])) ++p;
    const char *s = t.c_str() + p;
    char *end = nullptr;
    double v = std::strtod(s, &end);
    if (end == s) throw Error(FCFD_ERR_MESH, std::string("grid file: expected a number (") + what + ")");
    p += (size_t)(end - s);
    return (T)v;
  }
};

std::string strip(const std::string &s) {
  std::string o;
  for (char c : s)
    if (!std::isspace((unsigned char)c)) o.push_back(c);
  return o;
}

std::string unquote(const std::string &s) {
  std::string o;
  for (char c : s)
    if (c != '"' && c != '\'') o.push_back(c);
  return o;
}

// StringExplode (inputs.cc:363-376): split at any separator character, empty
// pieces dropped
std::vector<std::string> explode(const std::string &s, char sep) {
  std::vector<std::string> out;
  size_t b = 0;
  for (;;) {
    size_t e = s.find(sep, b);
    std::string piece = s.substr(b, e == std::string::npos ? std::string::npos : e - b);
    if (!piece.empty()) out.push_back(piece);
    if (e == std::string::npos) break;
    b = e + 1;
  }
  return out;
}

struct TecGrid {
  int n_nodes = 0, n_cells = 0, n_faces = 0;
  std::vector<double> xyz;
  std::vector<int32_t> f_index, f_nodes, left, right;
  std::vector<std::set<int32_t>> bc_nodes;
  std::vector<std::string> bc_names;
  std::vector<int32_t> c_index, c_nodes;
};

TecGrid read_tec(const std::string &path) {
  Cursor in;
  {
    std::ifstream f(path, std::ios::binary);
    if (!f.is_open()) throw Error(FCFD_ERR_INPUT, "grid file " + path + " could not be found");
    std::stringstream ss;
    ss << f.rdbuf();
    in.t = ss.str();
  }
  TecGrid g;
  std::string line;
  while (!in.first_numeric()) {
    if (!in.getline(line)) throw Error(FCFD_ERR_MESH, "error reading grid file " + path);
    for (const std::string &ex : explode(strip(line), ',')) {
      std::vector<std::string> kv = explode(ex, '=');
      if (kv.size() != 2) continue;
      if (kv[0] == "Nodes") g.n_nodes = std::atoi(kv[1].c_str());
      else if (kv[0] == "Elements") g.n_cells = std::atoi(kv[1].c_str());
      else if (kv[0] == "Faces") g.n_faces = std::atoi(kv[1].c_str());
      else if (kv[0] == "ZONETYPE" && kv[1] != "FEPolyhedron") throw Error(FCFD_ERR_UNSUPPORTED, "ZONETYPE=" + kv[1] + " is not supported");
      else if (kv[0] == "DATAPACKING" && kv[1] != "BLOCK") throw Error(FCFD_ERR_UNSUPPORTED, "DATAPACKING=" + kv[1] + " is not supported");
      else if (kv[0] == "NumConnectedBoundaryFaces" && std::atoi(kv[1].c_str()) != 0)
        throw Error(FCFD_ERR_UNSUPPORTED, "NumConnectedBoundaryFaces>0 is not supported");
      else if (kv[0] == "TotalNumBoundaryConnections" && std::atoi(kv[1].c_str()) != 0)
        throw Error(FCFD_ERR_UNSUPPORTED, "TotalNumBoundaryConnections>0 is not supported");
    }
  }
  if (g.n_nodes <= 0 || g.n_cells <= 0 || g.n_faces <= 0) throw Error(FCFD_ERR_MESH, "grid file header lacks Nodes, Elements or Faces");
  g.xyz.assign(3 * (size_t)g.n_nodes, 0.);
  for (int i = 0; i < 3; ++i)
    for (int n = 0; n < g.n_nodes; ++n) g.xyz[3 * (size_t)n + i] = in.number<double>("node coordinates");
  auto skip_comment = [&]() { if (!in.first_numeric()) in.getline(line); };
  skip_comment();
  g.f_index.assign(g.n_faces + 1, 0);
  for (int f = 0; f < g.n_faces; ++f) {
    const int k = in.number<int>("face node counts");
    if (k < 1) throw Error(FCFD_ERR_MESH, "grid file: face with no nodes");
    g.f_index[f + 1] = g.f_index[f] + k;
  }
  skip_comment();
  g.f_nodes.resize(g.f_index[g.n_faces]);
  for (auto &v : g.f_nodes) {
    v = in.number<int>("face nodes") - 1;
    if (v < 0 || v >= g.n_nodes) throw Error(FCFD_ERR_MESH, "grid file: face node out of range");
  }
  skip_comment();
  g.left.resize(g.n_faces);
  for (auto &v : g.left) v = in.number<int>("left elements") - 1;
  skip_comment();
  g.right.resize(g.n_faces);
  for (auto &v : g.right) v = in.number<int>("right elements") - 1;
  for (int f = 0; f < g.n_faces; ++f)
    if (g.left[f] >= g.n_cells || g.right[f] >= g.n_cells || g.left[f] < -1 || g.right[f] < -1)
      throw Error(FCFD_ERR_MESH, "grid file: face element out of range");
  // boundary nodes: the nodes of faces with a missing left or right element
  std::vector<char> on_boundary(g.n_nodes, 0);
  for (int f = 0; f < g.n_faces; ++f)
    if (g.left[f] < 0 || g.right[f] < 0)
      for (int k = g.f_index[f]; k < g.f_index[f + 1]; ++k) on_boundary[g.f_nodes[k]] = 1;
  struct KeyHash {
    size_t operator()(const std::array<uint64_t, 3> &k) const { return k[0] * 1000003u ^ k[1] * 7919u ^ k[2]; }
  };
  std::unordered_map<std::array<uint64_t, 3>, int, KeyHash> exact;
  std::vector<int> bnodes;
  for (int n = 0; n < g.n_nodes; ++n) {
    if (!on_boundary[n]) continue;
    bnodes.push_back(n);
    std::array<uint64_t, 3> k;
    std::memcpy(k.data(), &g.xyz[3 * (size_t)n], 24);
    exact.emplace(k, n);  // the lowest id among equal coordinates stays
  }
  auto nearest = [&](const double q[3]) {
    std::array<uint64_t, 3> k;
    std::memcpy(k.data(), q, 24);
    auto it = exact.find(k);
    if (it != exact.end()) return it->second;
    int best = -1;
    double bd = INFINITY;
    for (int n : bnodes) {
      const double *x = &g.xyz[3 * (size_t)n];
      const double d = (x[0] - q[0]) * (x[0] - q[0]) + (x[1] - q[1]) * (x[1] - q[1]) + (x[2] - q[2]) * (x[2] - q[2]);
      if (d < bd) { bd = d; best = n; }
    }
    return best;
  };
  // boundary zones (grid_reader_tec.cc:169-229)
  bool grabbed = false;
  while (true) {
    int zone_nodes = 0;
    while (true) {
      if (in.first_numeric()) break;
      if (!grabbed && !in.getline(line)) throw Error(FCFD_ERR_MESH, "error reading grid file " + path);
      grabbed = false;
      for (const std::string &ex : explode(strip(line), ',')) {
        std::vector<std::string> kv = explode(ex, '=');
        if (kv.size() != 2) continue;
        if (kv[0] == "ZONET") {
          g.bc_names.push_back(unquote(kv[1]));
          g.bc_nodes.emplace_back();
        } else if (kv[0] == "Nodes") {
          zone_nodes = std::atoi(kv[1].c_str());
        }
      }
    }
    if (g.bc_nodes.empty()) throw Error(FCFD_ERR_MESH, "grid file: boundary zone without a ZONE T= line");
    std::vector<double> zx(3 * (size_t)zone_nodes);
    for (int i = 0; i < 3; ++i)
      for (int n = 0; n < zone_nodes; ++n) zx[3 * (size_t)n + i] = in.number<double>("boundary zone coordinates");
    // a zone whose ZONE T= line was not read adds to the previous region, as
    // in the reference
    for (int n = 0; n < zone_nodes; ++n) {
      const int id = nearest(&zx[3 * (size_t)n]);
      if (id >= 0) g.bc_nodes.back().insert(id);
    }
    // skip to the next ZONE line or the end
    bool more = false;
    while (true) {
      const bool ok = in.getline(line);
      const std::string s = strip(line);
      if (s.compare(0, 4, "ZONE") == 0) { grabbed = true; more = true; break; }
      if (!ok || in.eof()) break;
    }
    if (!more) break;
  }
  // cell node lists: sorted node sets of their faces
  std::vector<std::set<int32_t>> cn(g.n_cells);
  for (int f = 0; f < g.n_faces; ++f)
    for (int k = g.f_index[f]; k < g.f_index[f + 1]; ++k) {
      if (g.left[f] >= 0) cn[g.left[f]].insert(g.f_nodes[k]);
      if (g.right[f] >= 0) cn[g.right[f]].insert(g.f_nodes[k]);
    }
  g.c_index.assign(g.n_cells + 1, 0);
  for (int c = 0; c < g.n_cells; ++c) {
    g.c_index[c + 1] = g.c_index[c] + (int)cn[c].size();
    g.c_nodes.insert(g.c_nodes.end(), cn[c].begin(), cn[c].end());
  }
  return g;
}

}  // namespace
}  // namespace fcfd

extern "C" {

int fcfd_mesh_from_tecplot(const char *path, const fcfd_case *cs, fcfd_mesh **out, char *bc_names, int32_t bc_names_len) {
  try {
    if (!path || !cs || !out) throw fcfd::Error(FCFD_ERR_INPUT, "null argument");
    fcfd::TecGrid g = fcfd::read_tec(path);
    std::vector<int32_t> bidx(1, 0), bnod;
    for (const auto &s : g.bc_nodes) {
      bnod.insert(bnod.end(), s.begin(), s.end());
      bidx.push_back((int32_t)bnod.size());
    }
    fcfd_raw_mesh raw{};
    raw.n_nodes = g.n_nodes;
    raw.xyz = g.xyz.data();
    raw.n_cells = g.n_cells;
    raw.conn_index = g.c_index.data();
    raw.conn = g.c_nodes.data();
    raw.n_bc = (int32_t)g.bc_nodes.size();
    raw.bc_index = bidx.data();
    raw.bc_nodes = bnod.data();
    fcfd::FaceInput fin;
    fin.n_faces = g.n_faces;
    fin.index = g.f_index.data();
    fin.nodes = g.f_nodes.data();
    fin.left = g.left.data();
    fin.right = g.right.data();
    fcfd_case copy = *cs;
    *out = fcfd::build_mesh(raw, copy, &fin);
    if (bc_names && bc_names_len > 0) {
      std::string all;
      for (size_t b = 0; b < g.bc_names.size(); ++b) all += (b ? "\n" : "") + g.bc_names[b];
      std::snprintf(bc_names, (size_t)bc_names_len, "%s", all.c_str());
    }
  } catch (const fcfd::Error &e) {
    fcfd::set_last_error(e.what());
    return e.code;
  } catch (const std::exception &e) {
    fcfd::set_last_error(e.what());
    return FCFD_ERR_MESH;
  }
  return FCFD_OK;
}

}  // extern "C"
