// Restart files in the reference's layout.
//
// write_restart (src/write_restart.cc:45-100) creates ./restart/ and
// ./restart/<step>/, writes the partition map ./restart/partitionMap_<gid>.dat
// (text: the partition count, then per partition "nodeCount\tcellCount" and
// one global cell id per line), <step>/time.dat (text, default stream
// formatting: the physical time; the three NS residual normalisations; the two
// RANS ones or "-1\t-1"; the heat-conduction one or "-1") and one raw
// native-endian file per cell variable (Variable::dump_cell_data,
// src/variable/variable.h:229-245): dt.<gid>, p.<gid>, V.<gid> (three doubles
// per cell), T.<gid> (ns_write_restart.cc:25-35) and k.<gid>, omega.<gid>,
// mu_t.<gid> (rans_write_restart.cc:25-35).  read_restart
// (src/read_restart.cc:44-102, Variable::read_cell_data variable.h:248-271)
// walks the partition map and places each value at the cell whose global id it
// names; here the mesh is one partition whose global id of cell c is c (the
// reference's cell order is kept), so files written by a partitioned run are
// scattered back by global id.
#include <sys/stat.h>

#include <cstdio>
#include <fstream>
#include <string>
#include <vector>

#include "internal.hpp"

namespace fcfd {
namespace {

std::string root_of(const char *dir) {
  std::string d = (dir && *dir) ? std::string(dir) : std::string(".");
  if (d.back() != '/') d += "/";
  return d;
}

// C++ default float formatting (precision 6, %g)
std::string g6(double v) {
  char b[64];
  std::snprintf(b, sizeof(b), "%g", v);
  return b;
}

void dump(const std::string &path, const double *v, size_t count) {
  std::ofstream f(path, std::ios::binary);
  if (!f.is_open()) throw Error(FCFD_ERR_INPUT, "restart file " + path + " could not be written");
  f.write(reinterpret_cast<const char *>(v), (std::streamsize)(sizeof(double) * count));
  if (!f.good()) throw Error(FCFD_ERR_INPUT, "restart file " + path + " could not be written");
}

// Variable::read_cell_data: `width` doubles per cell, in partition-map order
void scatter(const std::string &path, const std::vector<std::vector<int>> &pmap, int n_cells, int width, double *out,
             int stride, int offset) {
  std::ifstream f(path, std::ios::binary);
  if (!f.is_open()) throw Error(FCFD_ERR_INPUT, "restart file " + path + " could not be opened");
  std::vector<double> v(width);
  for (const auto &part : pmap)
    for (int gid : part) {
      f.read(reinterpret_cast<char *>(v.data()), (std::streamsize)(sizeof(double) * width));
      if (!f.good()) throw Error(FCFD_ERR_INPUT, "restart file " + path + " is shorter than its partition map");
      if (gid >= 0 && gid < n_cells)
        for (int k = 0; k < width; ++k) out[(size_t)gid * stride + offset + k] = v[k];
    }
}

}  // namespace

void restart_write(const char *dir, int gid, int step, double time, const double *first_res, const double *rans_first,
                   int n_cells, int n_nodes, const double *W, const double *dt, const double *K, const double *mu_t) {
  const std::string root = root_of(dir), rdir = root + "restart", sdir = rdir + "/" + std::to_string(step);
  mkdir(rdir.c_str(), S_IRWXU);
  mkdir(sdir.c_str(), S_IRWXU);
  const std::string gs = "." + std::to_string(gid);
  {
    std::ofstream f(rdir + "/partitionMap_" + std::to_string(gid) + ".dat");
    if (!f.is_open()) throw Error(FCFD_ERR_INPUT, "restart directory " + rdir + " could not be written");
    f << 1 << "\n" << n_nodes << "\t" << n_cells << "\n";
    for (int c = 0; c < n_cells; ++c) f << c << "\n";
  }
  {
    std::ofstream f(sdir + "/time.dat");
    if (!f.is_open()) throw Error(FCFD_ERR_INPUT, "restart directory " + sdir + " could not be written");
    f << g6(time) << "\n";
    f << g6(first_res[0]) << "\t" << g6(first_res[1]) << "\t" << g6(first_res[2]) << "\n";
    if (rans_first) f << g6(rans_first[0]) << "\t" << g6(rans_first[1]) << "\n";
    else f << "-1\t-1\n";
    f << "-1\n";
  }
  std::vector<double> a(n_cells), v3(3 * (size_t)n_cells);
  if (dt) dump(sdir + "/dt" + gs, dt, n_cells);
  for (int c = 0; c < n_cells; ++c) a[c] = W[5 * (size_t)c];
  dump(sdir + "/p" + gs, a.data(), n_cells);
  for (int c = 0; c < n_cells; ++c)
    for (int k = 0; k < 3; ++k) v3[3 * (size_t)c + k] = W[5 * (size_t)c + 1 + k];
  dump(sdir + "/V" + gs, v3.data(), v3.size());
  for (int c = 0; c < n_cells; ++c) a[c] = W[5 * (size_t)c + 4];
  dump(sdir + "/T" + gs, a.data(), n_cells);
  if (K) {
    for (int c = 0; c < n_cells; ++c) a[c] = K[2 * (size_t)c];
    dump(sdir + "/k" + gs, a.data(), n_cells);
    for (int c = 0; c < n_cells; ++c) a[c] = K[2 * (size_t)c + 1];
    dump(sdir + "/omega" + gs, a.data(), n_cells);
    if (mu_t) dump(sdir + "/mu_t" + gs, mu_t, n_cells);
  }
}

void restart_read(const char *dir, int gid, int step, int n_cells, double *time, double *first_res, double *rans_first,
                  double *W, double *K, double *mu_t) {
  const std::string root = root_of(dir), rdir = root + "restart", sdir = rdir + "/" + std::to_string(step);
  const std::string gs = "." + std::to_string(gid);
  std::vector<std::vector<int>> pmap;
  {
    const std::string fn = rdir + "/partitionMap_" + std::to_string(gid) + ".dat";
    std::ifstream f(fn);
    if (!f.is_open()) throw Error(FCFD_ERR_INPUT, "restart file " + fn + " couldn't be opened");
    int np = 0;
    f >> np;
    if (!f.good() || np < 1) throw Error(FCFD_ERR_INPUT, "restart file " + fn + " has no partition count");
    pmap.resize(np);
    for (int p = 0; p < np; ++p) {
      int nn = 0, ncp = 0;
      f >> nn >> ncp;
      if (!f.good() || ncp < 0) throw Error(FCFD_ERR_INPUT, "restart file " + fn + " is truncated");
      pmap[p].resize(ncp);
      for (int c = 0; c < ncp; ++c) f >> pmap[p][c];
      if (f.fail()) throw Error(FCFD_ERR_INPUT, "restart file " + fn + " is truncated");
    }
    size_t total = 0;
    for (const auto &q : pmap) total += q.size();
    if ((int)total != n_cells) throw Error(FCFD_ERR_INPUT, "restart partition map holds " + std::to_string(total) +
                                                               " cells, the mesh " + std::to_string(n_cells));
  }
  {
    std::ifstream f(sdir + "/time.dat");
    if (!f.is_open()) throw Error(FCFD_ERR_INPUT, "restart file " + sdir + "/time.dat couldn't be opened");
    double t = 0., r[3] = {0., 0., 0.}, q[2] = {-1., -1.};
    f >> t >> r[0] >> r[1] >> r[2] >> q[0] >> q[1];
    if (f.fail()) throw Error(FCFD_ERR_INPUT, "restart file " + sdir + "/time.dat is truncated");
    if (time) *time = t;
    if (first_res)
      for (int k = 0; k < 3; ++k) first_res[k] = r[k];
    if (rans_first) { rans_first[0] = q[0]; rans_first[1] = q[1]; }
  }
  scatter(sdir + "/p" + gs, pmap, n_cells, 1, W, 5, 0);
  scatter(sdir + "/V" + gs, pmap, n_cells, 3, W, 5, 1);
  scatter(sdir + "/T" + gs, pmap, n_cells, 1, W, 5, 4);
  if (K) {
    scatter(sdir + "/k" + gs, pmap, n_cells, 1, K, 2, 0);
    scatter(sdir + "/omega" + gs, pmap, n_cells, 1, K, 2, 1);
  }
  if (mu_t) scatter(sdir + "/mu_t" + gs, pmap, n_cells, 1, mu_t, 1, 0);
}

}  // namespace fcfd

extern "C" {

int fcfd_restart_write(const char *dir, int32_t gid, int32_t step, double time, const double *first_res,
                       const double *rans_first_res, int32_t n_cells, int32_t n_nodes, const double *W, const double *dt,
                       const double *K, const double *mu_t) {
  try {
    if (!first_res || !W || n_cells < 0) throw fcfd::Error(FCFD_ERR_INPUT, "null argument");
    fcfd::restart_write(dir, gid, step, time, first_res, rans_first_res, n_cells, n_nodes, W, dt, K, mu_t);
  } catch (const fcfd::Error &e) {
    fcfd::set_last_error(e.what());
    return e.code;
  }
  return FCFD_OK;
}

int fcfd_restart_read(const char *dir, int32_t gid, int32_t step, int32_t n_cells, double *time, double *first_res,
                      double *rans_first_res, double *W, double *K, double *mu_t) {
  try {
    if (!W || n_cells < 0) throw fcfd::Error(FCFD_ERR_INPUT, "null argument");
    fcfd::restart_read(dir, gid, step, n_cells, time, first_res, rans_first_res, W, K, mu_t);
  } catch (const fcfd::Error &e) {
    fcfd::set_last_error(e.what());
    return e.code;
  }
  return FCFD_OK;
}

}  // extern "C"
