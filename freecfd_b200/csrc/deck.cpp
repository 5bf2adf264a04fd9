// Input-deck reader for the residual path.
//
// Reads the reference's deck format with the reference's semantics
// (src/inputs/inputs.cc:37-345): comments are dropped, then every whitespace
// character is removed; a section is `name{...}` (numbered `name_N{...}`), a
// subsection `name(...);`, an entry `key=value;` whose key must follow one of
// `({;` or start the text.  Each successful lookup consumes the text it
// matched, subsections are taken out of their section before the section's own
// entries are read, and keys are looked up in sorted order per value type —
// so a deck reads the same here as in the reference.  Names and defaults follow
// src/read_inputs.cc:28-218; the material file follows read_inputs.cc:181-215
// and MATERIAL::set (src/material/material.cc:29-106); BC values follow
// NavierStokes::set_bcs (src/navier_stokes/ns_set_bcs.cc:25-140).
#include <cstdlib>
#include <fstream>
#include <map>
#include <sstream>

#include "internal.hpp"

namespace fcfd {
namespace {

// Find `open`...`close` after a character from `accept` (or at position 0),
// return the text between and cut the whole match out of `text`.
bool take(std::string &text, const std::string &open, const std::string &close, std::string &out,
          bool check_before = false, const char *accept = "") {
  size_t from = 0;
  for (;;) {
    size_t b = text.find(open, from);
    if (b == std::string::npos) return false;
    size_t e = text.find(close, b + open.size());
    if (e == std::string::npos) return false;
    bool ok = !check_before || b == 0 || std::string(accept).find(text[b - 1]) != std::string::npos;
    if (ok) {
      out = text.substr(b + open.size(), e - b - open.size());
      text.erase(b, e + close.size() - b);
      return true;
    }
    from = e;  // resume after the rejected candidate's terminator
  }
}

int count_of(const std::string &hay, const std::string &needle) {
  int n = 0;
  for (size_t p = hay.find(needle); p != std::string::npos; p = hay.find(needle, p + needle.size())) ++n;
  return n;
}

std::string clean(const std::string &raw) {
  std::string t = raw, dummy;
  while (take(t, "/*", "*/", dummy)) {}
  while (take(t, "//", "\n", dummy)) {}
  std::string out;
  out.reserve(t.size());
  for (char ch : t)
    if (ch != ' ' && ch != '\t' && ch != '\f' && ch != '\v' && ch != '\n' && ch != '\r') out.push_back(ch);
  return out;
}

// A block of entries with a typed, sorted key registry.
struct Block {
  std::string text;
  bool found = false;
  struct D { double v; bool found; };
  struct S { std::string v; bool found; };
  struct V { double v[3]; bool found; };
  std::map<std::string, std::pair<bool, int>> ireg;         // key -> (required, default)
  std::map<std::string, std::pair<bool, double>> dreg;
  std::map<std::string, std::pair<bool, std::string>> sreg;
  std::map<std::string, std::pair<bool, double>> vreg;
  std::map<std::string, bool> slreg;                        // string lists (value unused here)
  std::map<std::string, int> iv;
  std::map<std::string, D> dv;
  std::map<std::string, S> sv;
  std::map<std::string, V> vv;
  std::map<std::string, std::vector<std::string>> slv;     // string lists, split at ','
  std::string where;

  void need(const std::string &k) const { throw Error(FCFD_ERR_INPUT, "required input entry " + where + " -> " + k + " could not be found"); }
  void read() {
    std::string val;
    for (auto &r : ireg) {
      bool f = take(text, r.first + "=", ";", val, true, "({;");
      if (!f && r.second.first) need(r.first);
      iv[r.first] = f ? std::atoi(val.c_str()) : r.second.second;
    }
    for (auto &r : dreg) {
      bool f = take(text, r.first + "=", ";", val, true, "({;");
      if (!f && r.second.first) need(r.first);
      dv[r.first] = D{f ? std::strtod(val.c_str(), nullptr) : r.second.second, f};
    }
    for (auto &r : sreg) {
      bool f = take(text, r.first + "=", ";", val, true, "({;");
      if (!f && r.second.first) need(r.first);
      sv[r.first] = S{f ? val : r.second.second, f};
    }
    for (auto &r : vreg) {
      bool f = take(text, r.first + "=", ";", val, true, "({;");
      if (!f && r.second.first) need(r.first);
      V x{{r.second.second, r.second.second, r.second.second}, f};
      if (f) {
        char *end;
        x.v[0] = std::strtod(val.c_str() + 1, &end);
        x.v[1] = std::strtod(end + 1, &end);
        x.v[2] = std::strtod(end + 1, nullptr);
      }
      vv[r.first] = x;
    }
    for (auto &r : slreg) {
      bool f = take(text, r.first + "=[", "];", val, true, "({;");
      if (!f && r.second) need(r.first);
      std::vector<std::string> items;
      if (f) {
        size_t b = 0;
        for (;;) {
          size_t e = val.find(',', b);
          items.push_back(val.substr(b, e == std::string::npos ? std::string::npos : e - b));
          if (e == std::string::npos) break;
          b = e + 1;
        }
      }
      slv[r.first] = items;
    }
  }
  double d(const std::string &k) const { return dv.at(k).v; }
  bool has(const std::string &k) const { auto it = dv.find(k); return it != dv.end() && it->second.found; }
  const std::string &s(const std::string &k) const { return sv.at(k).v; }
  bool has_s(const std::string &k) const { auto it = sv.find(k); return it != sv.end() && it->second.found; }
  int i(const std::string &k) const { return iv.at(k); }
};

struct Sub : Block {};

// A section with its subsections (single and numbered), read like the reference:
// single subsections (sorted), numbered subsections (sorted), then own entries.
struct Sec : Block {
  std::map<std::string, Sub> subs;
  std::map<std::string, std::vector<Sub>> nsubs;
  std::map<std::string, Sub> nsub_tmpl;
  void read_from(std::string &file_text, const std::string &full_name, bool required) {
    found = take(file_text, full_name + "{", "}", text, true, "};");
    if (required && !found) throw Error(FCFD_ERR_INPUT, "required input section " + full_name + " could not be found");
    for (auto &kv : subs) {
      kv.second.where = where + " -> " + kv.first;
      kv.second.found = take(text, kv.first + "(", ");", kv.second.text, true, "};");
      kv.second.read();
    }
    for (auto &kv : nsub_tmpl) {
      int n = count_of(text, kv.first + "_");
      auto &vec = nsubs[kv.first];
      vec.assign(n, kv.second);
      for (int k = 0; k < n; ++k) {
        std::string nm = kv.first + "_" + std::to_string(k + 1);
        vec[k].where = where + " -> " + nm;
        vec[k].found = take(text, nm + "(", ");", vec[k].text, true, "};");
        vec[k].read();
      }
    }
    read();
  }
};

std::string slurp(const std::string &path) {
  std::ifstream f(path);
  if (!f.is_open()) throw Error(FCFD_ERR_INPUT, "input file " + path + " could not be found");
  std::stringstream ss;
  std::string line, all;
  while (std::getline(f, line)) all += line + "\n";
  return all;
}

int grad_method(const std::string &s) {
  if (s == "lsqr") return GM_LSQR;
  if (s == "greengauss") return GM_GREENGAUSS;
  return GM_CURVILINEAR;
}

// timemarching and pseudotime sections (read_inputs.cc:152-176) and the step
// type logic of set_time_step_options (time_step.cc:25-60)
TimeMarching parse_time_marching(std::string &text) {
  const bool req = true, opt = false;
  Sec tm;
  tm.where = "timemarching";
  tm.sreg = {{"integrator", {opt, "backwardEuler"}}, {"schedulefile", {opt, "none"}}};
  tm.dreg = {{"stepsize", {opt, 1.}}, {"CFLmax", {opt, 1000.}}, {"CFLlocal", {opt, 1000.}}};
  tm.ireg = {{"numberofsteps", {req, 0}}, {"updatefrequency", {opt, 1000000}}};
  Sub ramp; ramp.dreg = {{"initial", {opt, 1.}}, {"growth", {opt, 1.2}}};
  tm.subs = {{"ramp", ramp}};
  tm.read_from(text, "timemarching", true);
  Sec ps;
  ps.where = "pseudotime";
  ps.sreg = {{"preconditioner", {opt, "none"}}};
  ps.dreg = {{"residualtolerance", {opt, 1e-8}}, {"stepsize", {opt, 1.}}, {"CFLmax", {opt, 1000.}}, {"CFLlocal", {opt, 1000.}}};
  ps.ireg = {{"numberofsteps", {opt, 1}}, {"updatefrequency", {opt, 1000000}}};
  Sub psramp; psramp.dreg = {{"initial", {opt, 1.}}, {"growth", {opt, 1.2}}};
  ps.subs = {{"ramp", psramp}};
  ps.read_from(text, "pseudotime", false);
  TimeMarching t;
  t.n_steps = tm.i("numberofsteps");
  t.update_freq = tm.i("updatefrequency");
  t.ramp = tm.subs["ramp"].found;
  t.ramp_initial = tm.subs["ramp"].d("initial");
  t.ramp_growth = tm.subs["ramp"].d("growth");
  t.stepsize = tm.d("stepsize");
  t.cfl_max = tm.d("CFLmax");
  t.cfl_local = tm.d("CFLlocal");
  if (tm.has("stepsize")) t.type = TS_FIXED;
  if (tm.has("CFLmax")) {
    if (t.type == TS_FIXED) throw Error(FCFD_ERR_INPUT, "input entry timemarching -> CFLmax can't be specified together with stepsize");
    t.type = TS_CFL_MAX;
  } else if (tm.has("CFLlocal")) {
    if (t.type == TS_FIXED) throw Error(FCFD_ERR_INPUT, "input entry timemarching -> CFLlocal can't be specified together with stepsize");
    t.type = TS_CFL_LOCAL;
  }
  if (tm.has_s("schedulefile")) t.schedule_file = tm.s("schedulefile");
  t.ps_steps = ps.i("numberofsteps");
  return t;
}

}  // namespace

TimeMarching read_time_marching(const std::string &path) {
  std::string text = clean(slurp(path));
  return parse_time_marching(text);
}

fcfd_case *read_deck(const std::string &path) {
  const bool req = true, opt = false;
  std::string text = clean(slurp(path));
  std::string dir;
  size_t slash = path.find_last_of('/');
  if (slash != std::string::npos) dir = path.substr(0, slash + 1);

  Sec ref;
  ref.where = "reference";
  ref.dreg = {{"p", {opt, 0.}}, {"T", {opt, 0.}}, {"Mach", {opt, 1.}}};
  ref.read_from(text, "reference", false);

  Sec grid;
  grid.where = "grid_1";
  grid.sreg = {{"file", {req, ""}}, {"format", {opt, "cgns"}}, {"equations", {req, ""}}, {"material", {opt, "none"}}};
  grid.ireg = {{"dimension", {opt, 3}}};
  Sub gradients; gradients.sreg = {{"hexmethod", {opt, "curvilinear"}}, {"prismmethod", {opt, "curvilinear"}}, {"othermethod", {opt, "lsqr"}}};
  Sub interp; interp.sreg = {{"method", {opt, "wtli"}}}; interp.ireg = {{"stencilsize", {opt, 2}}}; interp.dreg = {{"skewnesstolerance", {opt, 0.99}}};
  Sub wout;
  wout.sreg = {{"format", {opt, "tecplot"}}};
  wout.ireg = {{"volumeplotfrequency", {opt, 1000000}}, {"surfaceplotfrequency", {opt, 1000000}}, {"restartfrequency", {opt, 1000000}}, {"loadfrequency", {opt, 1000000}}};
  wout.vreg = {{"momentcenter", {opt, 0.}}};
  wout.slreg = {{"includebcs", opt}, {"volumevariables", req}, {"surfacevariables", req}};
  Sub mat;
  mat.dreg = {{"gamma", {opt, 1.4}}, {"molarmass", {opt, 28.97}}, {"viscosity", {opt, 0.}}, {"thermalconductivity", {opt, 0.}}, {"Cp", {opt, 1000.}}, {"density", {opt, 0.}}};
  Sub turb;
  turb.dreg = {{"relativetolerance", {opt, 1e-6}}, {"absolutetolerance", {opt, 1e-12}}, {"klowlimit", {opt, 1e-10}}, {"khighlimit", {opt, 1e8}},
               {"omegalowlimit", {opt, 1e-2}}, {"viscosityratiolimit", {opt, 1e8}}, {"turbulentPr", {opt, 0.9}}};
  turb.ireg = {{"maximumiterations", {opt, 10}}};
  turb.sreg = {{"model", {opt, "sst"}}};
  Sub ns;
  ns.dreg = {{"relativetolerance", {opt, 1e-6}}, {"absolutetolerance", {opt, 1e-12}}, {"limiterthreshold", {opt, 0.}}, {"walldissipation", {opt, 0.3}}, {"BLheight", {opt, 0.}}};
  ns.ireg = {{"maximumiterations", {opt, 10}}};
  ns.sreg = {{"limiter", {opt, "vk"}}, {"order", {opt, "second"}}, {"jacobianorder", {opt, "first"}}, {"convectiveflux", {opt, "AUSM+up"}}};
  Sub hc; hc.dreg = {{"relativetolerance", {opt, 1e-6}}, {"absolutetolerance", {opt, 1e-12}}}; hc.ireg = {{"maximumiterations", {opt, 10}}};
  grid.subs = {{"gradients", gradients}, {"interpolation", interp}, {"writeoutput", wout}, {"material", mat},
               {"turbulence", turb}, {"navierstokes", ns}, {"heatconduction", hc}};
  Sub ic;
  ic.sreg = {{"region", {opt, "box"}}, {"gradienttest", {opt, "none"}}};
  ic.vreg = {{"corner_1", {opt, -1e20}}, {"corner_2", {opt, 1e20}}, {"center", {opt, 0.}}, {"axisdirection", {opt, 0.}}, {"V", {opt, 0.}}};
  ic.dreg = {{"radius", {opt, 0.}}, {"height", {opt, 0.}}, {"p", {opt, 0.}}, {"T", {opt, 0.}}, {"rho", {opt, 0.}},
             {"turbulenceintensity", {opt, 1e-4}}, {"eddyviscosityratio", {opt, 0.1}}, {"BLthickness", {opt, -1.}}};
  Sub bcs;
  bcs.sreg = {{"type", {req, ""}}, {"kind", {opt, "none"}}, {"region", {opt, "gridfile"}}, {"interface", {opt, "none"}}, {"pick", {opt, "override"}}};
  bcs.vreg = {{"corner_1", {opt, 0.}}, {"corner_2", {opt, 0.}}, {"V", {opt, 0.}}};
  bcs.dreg = {{"p", {opt, 0.}}, {"p_total", {opt, 0.}}, {"mdot", {opt, 0.}}, {"qdot", {opt, 0.}}, {"T", {opt, 0.}}, {"T_total", {opt, 0.}},
              {"rho", {opt, 0.}}, {"turbulenceintensity", {opt, 1e-4}}, {"eddyviscosityratio", {opt, 0.1}}};
  Sub tr;
  tr.sreg = {{"function", {opt, ""}}};
  tr.vreg = {{"anchor", {opt, 0.}}, {"end", {opt, 0.}}, {"factor", {opt, 0.}}, {"axis", {opt, 0.}}};
  tr.dreg = {{"angle", {opt, 0.}}};
  grid.nsub_tmpl = {{"BC", bcs}, {"IC", ic}, {"transform", tr}};
  int ngrids = count_of(text, "grid_");
  if (ngrids < 1) throw Error(FCFD_ERR_INPUT, "required input section grid_1 could not be found");
  if (ngrids > 1) throw Error(FCFD_ERR_UNSUPPORTED, "multi-grid decks are outside the residual path");
  grid.read_from(text, "grid_1", true);

  const TimeMarching tmo = parse_time_marching(text);

  auto cs = new fcfd_case();
  try {
    cs->tm = tmo;
    cs->deck_path = path;
    {
      const Sub &wo = grid.subs["writeoutput"];
      cs->restart_freq = wo.i("restartfrequency");
      cs->load_freq = wo.i("loadfrequency");
      for (int k = 0; k < 3; ++k) cs->moment_center[k] = wo.vv.at("momentcenter").v[k];
      for (const std::string &b : wo.slv.at("includebcs")) cs->load_bcs.push_back(std::atoi(b.c_str()) - 1);
      const Sub &nsl = grid.subs["navierstokes"];
      cs->lin_rtol = nsl.d("relativetolerance");
      cs->lin_abstol = nsl.d("absolutetolerance");
      cs->lin_maxits = nsl.i("maximumiterations");
    }
    cs->dimension = grid.i("dimension");
    const Sub &nss = grid.subs["navierstokes"];
    const std::string &lim = nss.s("limiter");
    cs->limiter = lim == "vk" ? LIM_VK : lim == "bj" ? LIM_BJ : lim == "minmod" ? LIM_MINMOD : LIM_NONE;
    cs->limiter_threshold = nss.d("limiterthreshold");
    if (nss.s("order") == "first") cs->order = ORDER_FIRST;
    else if (nss.s("order") == "second") cs->order = ORDER_SECOND;
    const std::string &fl = nss.s("convectiveflux");
    if (fl == "AUSM+up") cs->flux = FLUX_AUSM_PLUS_UP;
    else if (fl == "Roe") cs->flux = FLUX_ROE;
    else if (fl == "vanLeer") cs->flux = FLUX_VAN_LEER;
    else if (fl == "SD-SLAU") cs->flux = FLUX_SD_SLAU;
    else if (fl == "SW") cs->flux = FLUX_SW;
    else throw Error(FCFD_ERR_UNSUPPORTED, "convective flux " + fl + " is not on the B200 path (Roe, AUSM+up, vanLeer, SD-SLAU, SW)");
    cs->wdiss = nss.d("walldissipation");
    cs->bl_height = nss.d("BLheight");
    cs->Minf = ref.d("Mach");
    cs->hex_method = grad_method(grid.subs["gradients"].s("hexmethod"));
    cs->prism_method = grad_method(grid.subs["gradients"].s("prismmethod"));
    cs->other_method = grad_method(grid.subs["gradients"].s("othermethod"));
    const std::string &im = grid.subs["interpolation"].s("method");
    cs->interp = im == "idw" ? IP_IDW : im == "simple" ? IP_SIMPLE : IP_WTLI;
    cs->stencil_size = grid.subs["interpolation"].i("stencilsize");
    cs->has_cfl_max = tmo.type == TS_CFL_MAX;
    cs->has_cfl_local = tmo.type == TS_CFL_LOCAL;
    cs->cfl_max = tmo.cfl_max;
    cs->cfl_local = tmo.cfl_local;
    const Sub &ts = grid.subs["turbulence"];
    cs->turbulent = ts.found;
    cs->turb_model = ts.s("model");
    cs->k_low = ts.d("klowlimit"); cs->k_high = ts.d("khighlimit"); cs->omega_low = ts.d("omegalowlimit");
    cs->visc_ratio_limit = ts.d("viscosityratiolimit"); cs->Pr_t = ts.d("turbulentPr");

    Material &m = cs->mat;
    if (grid.has_s("material")) {
      std::string mtext = clean(slurp(dir + grid.s("material") + ".mat"));
      Sec eos; eos.sreg = {{"model", {opt, "idealgas"}}}; eos.read_from(mtext, "equationofstate", false);
      Sec visc; visc.sreg = {{"model", {opt, "sutherlands"}}};
      visc.dreg = {{"referenceviscosity", {opt, 1.716e-5}}, {"referencetemperature", {opt, 273.15}}, {"sutherlandtemperature", {opt, 110.4}}};
      visc.read_from(mtext, "viscosity", false);
      Sec cp; cp.sreg = {{"model", {opt, "shomate"}}}; cp.ireg = {{"numberofpieces", {opt, 0}}}; cp.read_from(mtext, "Cp", false);
      Sec tc; tc.sreg = {{"model", {opt, "constantPrandtl"}}}; tc.dreg = {{"Pr", {opt, 0.7}}}; tc.read_from(mtext, "thermalconductivity", false);
      Block top; top.text = mtext;
      top.dreg = {{"molarmass", {opt, 28.97}}, {"density", {opt, 0.}}, {"gamma", {opt, 1.4}}, {"viscosity", {opt, 1.716e-5}},
                  {"Cp", {opt, 1000.}}, {"thermalconductivity", {opt, 0.024}}};
      top.read();
      m.Mw = top.d("molarmass");
      m.gamma = top.d("gamma");
      if (eos.s("model") != "idealgas") throw Error(FCFD_ERR_INPUT, "invalid equation of state option");
      m.R = 8314.47215 / m.Mw;
      if (top.has("viscosity")) { m.sutherland = false; m.mu = top.d("viscosity"); }
      else if (visc.found) {
        if (visc.s("model") != "sutherlands") throw Error(FCFD_ERR_INPUT, "invalid viscosity -> model option");
        m.sutherland = true;
        m.sut_mu_ref = visc.d("referenceviscosity"); m.sut_T_ref = visc.d("referencetemperature"); m.sut_S = visc.d("sutherlandtemperature");
      }
      if (top.has("thermalconductivity")) { m.prandtl = false; m.lambda = top.d("thermalconductivity"); }
      else if (tc.found) {
        if (tc.s("model") != "constantPrandtl") throw Error(FCFD_ERR_INPUT, "invalid thermalconductivity -> model option");
        m.prandtl = true;
        m.Pr = tc.d("Pr");
      }
    } else {
      const Sub &ms = grid.subs["material"];
      m.Mw = ms.d("molarmass");
      m.R = 8314.47215 / m.Mw;
      m.gamma = ms.d("gamma");
      m.sutherland = false;
      m.mu = ms.d("viscosity");
      m.prandtl = false;
      m.lambda = ms.d("thermalconductivity");
    }
    m.Pref = ref.d("p");
    m.Tref = ref.d("T");

    // BC regions: set_bcs.cc:46-86 (type/kind/box) and ns_set_bcs.cc:25-140 (values)
    const auto &bl = grid.nsubs["BC"];
    for (size_t b = 0; b < bl.size(); ++b) {
      const Sub &r = bl[b];
      BcRegion R;
      const std::string &type = r.s("type"), &kind = r.s("kind");
      if (type == "wall") R.type = BC_WALL;
      if (type == "inlet") R.type = BC_INLET;
      if (type == "outlet") R.type = BC_OUTLET;
      if (type == "symmetry") R.type = BC_SYMMETRY;
      if (kind == "slip") R.kind = K_SLIP;
      std::string pick = r.s("pick");
      if (pick.substr(0, 2) == "BC") { R.pick_from = std::atoi(pick.substr(2).c_str()); pick = "BC"; }
      R.pick = pick;
      R.box = (r.s("region") == "box");
      for (int k = 0; k < 3; ++k) { R.corner1[k] = r.vv.at("corner_1").v[k]; R.corner2[k] = r.vv.at("corner_2").v[k]; }
      if (kind == "none") R.kind = K_NONE;
      if (kind == "noreverse") R.kind = K_NO_REVERSE;
      if (kind == "dampreverse") R.kind = K_DAMP_REVERSE;
      if (kind == "slip") R.kind = K_SLIP;
      if (kind == "forcesupersonic") R.kind = K_FORCE_SUPERSONIC;
      if (r.has("p_total") && r.has("T_total")) { R.kind = K_STAGNATION; R.p_total = r.d("p_total"); R.T_total = r.d("T_total"); }
      auto rho_of = [&](double p, double T) { return (p + m.Pref) / (m.R * (T + m.Tref)); };
      auto T_of = [&](double p, double rho) { return (p + m.Pref) / (m.R * rho) - m.Tref; };
      auto p_of = [&](double rho, double T) { return rho * m.R * (T + m.Tref) - m.Pref; };
      if (r.has("p")) {
        R.p_fixed = true; R.p = r.d("p"); R.specified = SP_P;
        if (r.has("T")) {
          if (r.has("rho")) throw Error(FCFD_ERR_INPUT, "thermodynamic state is overspecified for BC_" + std::to_string(b + 1));
          R.T_fixed = true; R.T = r.d("T");
          R.rho_fixed = true; R.rho = rho_of(R.p, R.T);
          R.thermal = TH_FIXED_T; R.specified = SP_STATE;
        } else if (r.has("rho")) {
          R.rho_fixed = true; R.rho = r.d("rho");
          R.T_fixed = true; R.T = T_of(R.p, R.rho);
          R.thermal = TH_FIXED_T; R.specified = SP_STATE;
        } else if (R.type == BC_WALL) {
          R.thermal = TH_ADIABATIC;
        }
      } else if (r.has("T")) {
        R.T_fixed = true; R.T = r.d("T");
        R.thermal = TH_FIXED_T; R.specified = SP_T;
        if (r.has("rho")) {
          R.rho_fixed = true; R.rho = r.d("rho");
          R.p_fixed = true; R.p = p_of(R.rho, R.T);
          R.specified = SP_STATE;
        }
      } else if (r.has("rho")) {
        R.rho_fixed = true; R.rho = r.d("rho");
        R.specified = SP_RHO;
      } else if (R.type == BC_WALL) {
        R.thermal = TH_ADIABATIC;
      }
      if (r.has("qdot") && R.type == BC_WALL) {
        if (r.has("T")) throw Error(FCFD_ERR_INPUT, "can't specify both temperature and qdot for BC_" + std::to_string(b + 1));
        R.thermal = TH_FIXED_Q; R.qdot_fixed = true; R.qdot = r.d("qdot");
      }
      if (R.type == BC_WALL && R.kind != K_SLIP) { R.V_fixed = true; R.V[0] = R.V[1] = R.V[2] = 0.; }
      if (R.type == BC_SYMMETRY) R.thermal = TH_ADIABATIC;
      if (r.vv.at("V").found) {
        R.V_fixed = true;
        for (int k = 0; k < 3; ++k) R.V[k] = r.vv.at("V").v[k];
        R.kind = K_VELOCITY;
      }
      if (r.has("mdot")) { R.kind = K_MDOT; R.mdot_fixed = true; R.mdot = r.d("mdot"); }
      R.turb_intensity = r.d("turbulenceintensity");
      R.turb_ratio = r.d("eddyviscosityratio");
      cs->bc.push_back(R);
    }
    const auto &il = grid.nsubs["IC"];
    if (!il.empty()) {
      const Sub &r = il[0];
      cs->ic_has_p = r.has("p"); cs->ic_has_T = r.has("T"); cs->ic_has_rho = r.has("rho");
      cs->ic_p = r.d("p"); cs->ic_T = r.d("T"); cs->ic_rho = r.d("rho");
      for (int k = 0; k < 3; ++k) cs->ic_V[k] = r.vv.at("V").v[k];
    }
    if (cs->turbulent && cs->turb_model != "k-omega")
      throw Error(FCFD_ERR_UNSUPPORTED, "turbulence model " + cs->turb_model + " is not on the B200 path (k-omega)");
  } catch (...) {
    delete cs;
    throw;
  }
  return cs;
}

}  // namespace fcfd
