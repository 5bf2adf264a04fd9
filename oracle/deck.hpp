// Oracle (test infrastructure only): restatement of Free CFD's input-deck reader.
//
// Follows src/inputs/inputs.cc:37-345 and src/inputs/inputs.h:37-194:
//  * C/C++ comments are stripped and then ALL whitespace is removed
//    (inputs.cc:57-60, 302-316), so "navier stokes" becomes "navierstokes";
//  * sections are "name{...}" (numbered "name_N{...}"), subsections
//    "name(...);" (numbered "name_N(...);"), entries "key=value;";
//  * every lookup is extract_in_between() with a preceding-character check,
//    and a successful lookup REMOVES the matched text (inputs.cc:318-345);
//  * registered names are read in std::map (alphabetical) order, ints, then
//    doubles, strings, Vec3Ds, int/double/string lists (inputs.cc:150-300).
// The schema (names and defaults) is the one in src/read_inputs.cc:28-218.
#pragma once
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace orc {

struct DeckError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

// inputs.cc:318-345
inline bool extract_in_between(std::string &data, const std::string &begin, const std::string &end,
                               std::string &result, bool check_char_before = false,
                               const std::string &acceptList = "") {
  size_t begin_pos = 0, end_pos = 0;
  bool found = false;
  while (!found) {
    begin_pos = data.find(begin, end_pos);
    if (begin_pos == std::string::npos) return false;
    end_pos = data.find(end, begin_pos + begin.length());
    if (end_pos == std::string::npos) return false;
    if (check_char_before) {
      if (begin_pos == 0) {
        found = true;
      } else {
        std::string pre = data.substr(begin_pos - 1, 1);
        if (pre.find_first_of(acceptList) != std::string::npos) found = true;
      }
    } else {
      found = true;
    }
    if (found) {
      result = data.substr(begin_pos + begin.length(), end_pos - begin_pos - begin.length());
      data.replace(begin_pos, end_pos + end.length() - begin_pos, "");
    }
  }
  return true;
}

// inputs.cc:347-357
inline int number_of_occurances(const std::string &haystack, const std::string &needle) {
  int count = -1;
  size_t found = 0, start;
  while (found != std::string::npos) {
    count++;
    start = (count == 0) ? 0 : found + needle.length();
    found = haystack.find(needle, start);
  }
  return count;
}

// inputs.cc:359-372
inline void string_explode(std::string str, const std::string &sep, std::vector<std::string> *out) {
  size_t found = str.find_first_of(sep);
  while (found != std::string::npos) {
    if (found > 0) out->push_back(str.substr(0, found));
    str = str.substr(found + 1);
    found = str.find_first_of(sep);
  }
  if (str.length() > 0) out->push_back(str);
}

inline void strip_comments(std::string &data) {  // inputs.cc:302-306
  std::string dummy;
  while (extract_in_between(data, "/*", "*/", dummy)) {}
  while (extract_in_between(data, "//", "\n", dummy)) {}
}

inline void strip_white_spaces(std::string &data) {  // inputs.cc:308-316
  const std::string ws(" \t\f\v\n\r");
  std::string out;
  out.reserve(data.size());
  for (char ch : data)
    if (ws.find(ch) == std::string::npos) out.push_back(ch);
  data.swap(out);
}

template <class T>
struct Entry {
  T value{};
  T default_value{};
  bool is_found = false;
  bool is_required = false;
};

struct V3d {
  double c[3] = {0, 0, 0};
};

// InputBaseContainer (inputs.h:58-130)
struct Container {
  std::string rawData, name, parentName;
  int index = -1, parentIndex = -1;
  bool is_required = false, is_found = false;
  std::map<std::string, Entry<int>> ints;
  std::map<std::string, Entry<double>> doubles;
  std::map<std::string, Entry<std::string>> strings;
  std::map<std::string, Entry<V3d>> vecs;
  std::map<std::string, Entry<std::vector<int>>> intLists;
  std::map<std::string, Entry<std::vector<double>>> doubleLists;
  std::map<std::string, Entry<std::vector<std::string>>> stringLists;

  void reg_int(const std::string &n, bool req, int d = 0) { Entry<int> e; e.is_required = req; e.default_value = d; ints.insert({n, e}); }
  void reg_double(const std::string &n, bool req, double d = 0) { Entry<double> e; e.is_required = req; e.default_value = d; doubles.insert({n, e}); }
  void reg_string(const std::string &n, bool req, const std::string &d = "") { Entry<std::string> e; e.is_required = req; e.default_value = d; strings.insert({n, e}); }
  void reg_vec(const std::string &n, bool req, double d = 0) {
    // register_Vec3D: default_value=default_value[0] sets all three components (inputs.h:76-80)
    Entry<V3d> e; e.is_required = req; e.default_value.c[0] = e.default_value.c[1] = e.default_value.c[2] = d; vecs.insert({n, e});
  }
  void reg_stringList(const std::string &n, bool req, const std::string &d = " ") {
    Entry<std::vector<std::string>> e; e.is_required = req; e.default_value.push_back(d); stringLists.insert({n, e});
  }
  void reg_doubleList(const std::string &n, bool req, double d = 0) {
    Entry<std::vector<double>> e; e.is_required = req; e.default_value.push_back(d); doubleLists.insert({n, e});
  }

  [[noreturn]] void not_found(const std::string &var) const {
    std::string path;
    if (!name.empty()) path = name + " -> ";
    if (!parentName.empty()) path = parentName + " -> ";
    throw DeckError("required input entry " + path + var + " could not be found");
  }

  // inputs.cc:150-300
  void readEntries() {
    for (auto &kv : ints) {
      std::string v;
      kv.second.is_found = extract_in_between(rawData, kv.first + "=", ";", v, true, "({;");
      if (kv.second.is_found) kv.second.value = std::atoi(v.c_str());
      else if (kv.second.is_required) not_found(kv.first);
      else kv.second.value = kv.second.default_value;
    }
    for (auto &kv : doubles) {
      std::string v;
      kv.second.is_found = extract_in_between(rawData, kv.first + "=", ";", v, true, "({;");
      if (kv.second.is_found) kv.second.value = std::strtod(v.c_str(), nullptr);
      else if (kv.second.is_required) not_found(kv.first);
      else kv.second.value = kv.second.default_value;
    }
    for (auto &kv : strings) {
      std::string v;
      kv.second.is_found = extract_in_between(rawData, kv.first + "=", ";", v, true, "({;");
      if (kv.second.is_found) kv.second.value = v;
      else if (kv.second.is_required) not_found(kv.first);
      else kv.second.value = kv.second.default_value;
    }
    for (auto &kv : vecs) {
      std::string v;
      kv.second.is_found = extract_in_between(rawData, kv.first + "=", ";", v, true, "({;");
      if (kv.second.is_found) {
        char *pEnd;
        kv.second.value.c[0] = std::strtod(v.c_str() + 1, &pEnd);
        kv.second.value.c[1] = std::strtod(pEnd + 1, &pEnd);
        kv.second.value.c[2] = std::strtod(pEnd + 1, nullptr);
      } else if (kv.second.is_required) not_found(kv.first);
      else kv.second.value = kv.second.default_value;
    }
    for (auto &kv : intLists) {
      std::string v;
      std::vector<std::string> ex;
      kv.second.is_found = extract_in_between(rawData, kv.first + "=[", "];", v, true, "({;");
      if (kv.second.is_found) { string_explode(v, ",", &ex); for (auto &s : ex) kv.second.value.push_back(std::atoi(s.c_str())); }
      else if (kv.second.is_required) not_found(kv.first);
      else kv.second.value = kv.second.default_value;
    }
    for (auto &kv : doubleLists) {
      std::string v;
      std::vector<std::string> ex;
      kv.second.is_found = extract_in_between(rawData, kv.first + "=[", "];", v, true, "({;");
      if (kv.second.is_found) { string_explode(v, ",", &ex); for (auto &s : ex) kv.second.value.push_back(std::strtod(s.c_str(), nullptr)); }
      else if (kv.second.is_required) not_found(kv.first);
      else kv.second.value = kv.second.default_value;
    }
    for (auto &kv : stringLists) {
      std::string v;
      kv.second.is_found = extract_in_between(rawData, kv.first + "=[", "];", v, true, "({;");
      if (kv.second.is_found) string_explode(v, ",", &kv.second.value);
      else if (kv.second.is_required) not_found(kv.first);
      else kv.second.value = kv.second.default_value;
    }
  }

  const Entry<int> &gi(const std::string &n) { return ints[n]; }
  const Entry<double> &gd(const std::string &n) { return doubles[n]; }
  const Entry<std::string> &gs(const std::string &n) { return strings[n]; }
  const Entry<V3d> &gv(const std::string &n) { return vecs[n]; }
};

struct Subsection : Container {
  bool numbered = false;
  int count = 0;
};

struct Section : Container {
  std::map<std::string, Subsection> subsections;
  std::map<std::string, std::vector<Subsection>> numberedSubsections;
  bool numbered = false;
  int count = 0;
  void reg_sub(const std::string &n, bool numbered_, bool req) {
    Subsection t; t.numbered = numbered_; t.count = 0; t.is_required = req; t.name = n; t.parentName = name;
    if (numbered_) numberedSubsections.insert({n, std::vector<Subsection>{t}});
    else subsections.insert({n, t});
  }
  Subsection &sub(const std::string &n, int number = -1) {
    if (number >= 0) return numberedSubsections[n][number];
    return subsections[n];
  }
};

// InputFile (inputs.h:149-180, inputs.cc:37-148)
struct InputFile : Container {
  std::string fileName;
  std::map<std::string, Section> sections;
  std::map<std::string, std::vector<Section>> numberedSections;

  void setText(std::string raw) {
    rawData = std::move(raw);
    strip_comments(rawData);
    strip_white_spaces(rawData);
  }
  void setFile(const std::string &fn) {
    fileName = fn;
    std::ifstream f(fn);
    if (!f.is_open()) throw DeckError("input file " + fn + " could not be found");
    std::string line, raw;
    while (std::getline(f, line)) raw += line + "\n";
    setText(raw);
  }
  void reg_section(const std::string &n, bool numbered_, bool req) {
    Section t; t.is_required = req; t.name = n;
    if (numbered_) { t.numbered = true; t.count = 0; numberedSections.insert({n, std::vector<Section>{t}}); }
    else sections.insert({n, t});
  }
  Section &section(const std::string &n, int number = -1) {
    if (number >= 0) return numberedSections[n][number];
    return sections[n];
  }
  void read(const std::string &n, int number = -1) {
    if (number != -1) {
      int count = number_of_occurances(rawData, n + "_");
      section(n, 0).count = count;
      for (int i = 0; i < count; ++i) {
        numberedSections[n].push_back(numberedSections[n][0]);
        numberedSections[n][i].index = i;
        readSection(n, i);
      }
    } else {
      readSection(n, -1);
    }
  }
  void readSection(const std::string &n, int number) {
    std::string full = n;
    if (number >= 0) full += "_" + std::to_string(number + 1);
    Section &s = section(n, number);
    s.is_found = extract_in_between(rawData, full + "{", "}", s.rawData, true, "};");
    if (s.is_required && !s.is_found) throw DeckError("required input section " + full + " could not be found");
    for (auto &kv : s.subsections) { kv.second.parentIndex = number; readSubsection(s, kv.second); }
    for (auto &kv : s.numberedSubsections) {
      int count = number_of_occurances(s.rawData, kv.first + "_");
      kv.second[0].count = count;
      for (int i = 1; i < count; ++i) kv.second.push_back(kv.second[0]);
      for (int i = 0; i < count; ++i) {
        kv.second[i].name += "_" + std::to_string(i + 1);
        kv.second[i].parentIndex = number;
        readSubsection(s, kv.second[i]);
      }
    }
    s.readEntries();
  }
  void readSubsection(Section &parent, Subsection &sub) {
    sub.is_found = extract_in_between(parent.rawData, sub.name + "(", ");", sub.rawData, true, "};");
    if (sub.is_required && !sub.is_found) throw DeckError("required input subsection " + sub.parentName + " -> " + sub.name + " could not be found");
    sub.readEntries();
  }
};

// read_inputs.cc:28-178 (the part of the schema the residual path reads)
inline void register_deck_schema(InputFile &in) {
  const bool req = true, opt = false, numbered = true, single = false;
  in.reg_section("reference", single, opt);
  Section &ref = in.section("reference");
  ref.reg_double("p", opt, 0.); ref.reg_double("T", opt, 0.); ref.reg_double("Mach", opt, 1.);
  in.read("reference");

  in.reg_section("grid", numbered, req);
  Section &g = in.section("grid", 0);
  g.reg_string("file", req); g.reg_string("format", opt, "cgns"); g.reg_int("dimension", opt, 3); g.reg_string("equations", req);
  g.reg_sub("gradients", single, opt);
  g.sub("gradients").reg_string("hexmethod", opt, "curvilinear");
  g.sub("gradients").reg_string("prismmethod", opt, "curvilinear");
  g.sub("gradients").reg_string("othermethod", opt, "lsqr");
  g.reg_sub("interpolation", single, opt);
  g.sub("interpolation").reg_string("method", opt, "wtli");
  g.sub("interpolation").reg_int("stencilsize", opt, 2);
  g.sub("interpolation").reg_double("skewnesstolerance", opt, 0.99);
  g.reg_sub("writeoutput", single, req);
  {
    Subsection &w = g.sub("writeoutput");
    w.reg_string("format", opt, "tecplot");
    w.reg_int("volumeplotfrequency", opt, 1000000); w.reg_int("surfaceplotfrequency", opt, 1000000);
    w.reg_int("restartfrequency", opt, 1000000); w.reg_int("loadfrequency", opt, 1000000);
    w.reg_vec("momentcenter", opt, 0.);
    w.reg_stringList("includebcs", opt); w.reg_stringList("volumevariables", req); w.reg_stringList("surfacevariables", req);
  }
  g.reg_string("material", opt, "none");
  g.reg_sub("material", single, opt);
  {
    Subsection &m = g.sub("material");
    m.reg_double("gamma", opt, 1.4); m.reg_double("molarmass", opt, 28.97); m.reg_double("viscosity", opt, 0.);
    m.reg_double("thermalconductivity", opt, 0.); m.reg_double("Cp", opt, 1000.); m.reg_double("density", opt, 0.);
  }
  g.reg_sub("IC", numbered, req);
  {
    Subsection &ic = g.sub("IC", 0);
    ic.reg_string("region", opt, "box"); ic.reg_vec("corner_1", opt, -1.e20); ic.reg_vec("corner_2", opt, 1e20);
    ic.reg_vec("center", opt); ic.reg_vec("axisdirection", opt); ic.reg_double("radius", opt); ic.reg_double("height", opt);
    ic.reg_double("p", opt); ic.reg_vec("V", opt); ic.reg_double("T", opt); ic.reg_double("rho", opt);
    ic.reg_double("turbulenceintensity", opt, 1.e-4); ic.reg_double("eddyviscosityratio", opt, 0.1);
    ic.reg_double("BLthickness", opt, -1.); ic.reg_string("gradienttest", opt, "none");
  }
  g.reg_sub("BC", numbered, req);
  {
    Subsection &bc = g.sub("BC", 0);
    bc.reg_string("type", req); bc.reg_string("kind", opt, "none"); bc.reg_string("region", opt, "gridfile");
    bc.reg_string("interface", opt, "none"); bc.reg_vec("corner_1", opt); bc.reg_vec("corner_2", opt);
    bc.reg_string("pick", opt, "override");
    bc.reg_double("p", opt); bc.reg_double("p_total", opt); bc.reg_double("mdot", opt); bc.reg_double("qdot", opt);
    bc.reg_vec("V", opt); bc.reg_double("T", opt); bc.reg_double("T_total", opt); bc.reg_double("rho", opt);
    bc.reg_double("turbulenceintensity", opt, 1.e-4); bc.reg_double("eddyviscosityratio", opt, 0.1);
  }
  g.reg_sub("turbulence", single, opt);
  {
    Subsection &t = g.sub("turbulence");
    t.reg_double("relativetolerance", opt, 1.e-6); t.reg_double("absolutetolerance", opt, 1.e-12);
    t.reg_int("maximumiterations", opt, 10); t.reg_string("model", opt, "sst");
    t.reg_double("klowlimit", opt, 1.e-10); t.reg_double("khighlimit", opt, 1.e8); t.reg_double("omegalowlimit", opt, 1.e-2);
    t.reg_double("viscosityratiolimit", opt, 1.e8); t.reg_double("turbulentPr", opt, 0.9);
  }
  g.reg_sub("navierstokes", single, opt);
  {
    Subsection &n = g.sub("navierstokes");
    n.reg_double("relativetolerance", opt, 1.e-6); n.reg_double("absolutetolerance", opt, 1.e-12);
    n.reg_int("maximumiterations", opt, 10); n.reg_string("limiter", opt, "vk"); n.reg_double("limiterthreshold", opt, 0.);
    n.reg_string("order", opt, "second"); n.reg_string("jacobianorder", opt, "first"); n.reg_string("convectiveflux", opt, "AUSM+up");
    n.reg_double("walldissipation", opt, 0.3); n.reg_double("BLheight", opt, 0.);
  }
  g.reg_sub("heatconduction", single, opt);
  g.reg_sub("transform", numbered, opt);
  in.read("grid", 0);

  in.reg_section("timemarching", single, req);
  Section &tm = in.section("timemarching");
  tm.reg_string("integrator", opt, "backwardEuler"); tm.reg_double("stepsize", opt, 1.);
  tm.reg_double("CFLmax", opt, 1000.); tm.reg_double("CFLlocal", opt, 1000.);
  tm.reg_sub("ramp", single, opt); tm.sub("ramp").reg_double("initial", opt, 1.); tm.sub("ramp").reg_double("growth", opt, 1.2);
  tm.reg_int("numberofsteps", req); tm.reg_int("updatefrequency", opt, 1000000); tm.reg_string("schedulefile", opt, "none");
  in.read("timemarching");

  in.reg_section("pseudotime", single, opt);
  Section &ps = in.section("pseudotime");
  ps.reg_string("preconditioner", opt, "none"); ps.reg_double("residualtolerance", opt, 1.e-8);
  ps.reg_double("stepsize", opt, 1.); ps.reg_double("CFLmax", opt, 1000.); ps.reg_double("CFLlocal", opt, 1000.);
  ps.reg_sub("ramp", single, opt); ps.sub("ramp").reg_double("initial", opt, 1.); ps.sub("ramp").reg_double("growth", opt, 1.2);
  ps.reg_int("numberofsteps", opt, 1); ps.reg_int("updatefrequency", opt, 1000000);
  in.read("pseudotime");
  in.readEntries();
}

// read_inputs.cc:181-215 (material file schema)
inline void register_material_schema(InputFile &m) {
  const bool opt = false, single = false;
  m.reg_double("molarmass", opt, 28.97);
  m.reg_double("density", opt, 0.);
  m.reg_double("gamma", opt, 1.4);
  m.reg_section("equationofstate", single, opt);
  m.section("equationofstate").reg_string("model", opt, "idealgas");
  m.read("equationofstate");
  m.reg_double("viscosity", opt, 1.716e-5);
  m.reg_section("viscosity", single, opt);
  m.section("viscosity").reg_string("model", opt, "sutherlands");
  m.section("viscosity").reg_double("referenceviscosity", opt, 1.716e-5);
  m.section("viscosity").reg_double("referencetemperature", opt, 273.15);
  m.section("viscosity").reg_double("sutherlandtemperature", opt, 110.4);
  m.read("viscosity");
  m.reg_double("Cp", opt, 1000.);
  m.reg_section("Cp", single, opt);
  m.section("Cp").reg_int("numberofpieces", opt);
  m.section("Cp").reg_string("model", opt, "shomate");
  m.section("Cp").reg_doubleList("coefficients", opt);
  m.read("Cp");
  m.reg_double("thermalconductivity", opt, 0.024);
  m.reg_section("thermalconductivity", single, opt);
  m.section("thermalconductivity").reg_string("model", opt, "constantPrandtl");
  m.section("thermalconductivity").reg_double("Pr", opt, 0.7);
  m.read("thermalconductivity");
  m.readEntries();
}

}  // namespace orc
