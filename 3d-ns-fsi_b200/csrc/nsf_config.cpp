// ConfigFile reader for the C ABI (nsf_config_load / nsf_config_parse / nsf_config_defaults).
//
// Replaces ConfigSettings::loadSettings / readSettingValues / setDerivedParameters
// (src/ConfigSettings.cpp:18-163), which use libconfig++. The file syntax is libconfig's: `name = value`
// (or `name : value`), optional `;`/`,` terminators, comments (`//`, `#`, `/* */`), integers, floats (with
// a decimal point or exponent), booleans, strings, arrays `[..]`, lists `(..)` and groups `{..}`.
// Typing is strict as in the reference: an integer setting read as float (or the reverse) is a
// configuration error ("Integers must NOT have a decimal point", ConfigSettings.cpp:131-135).
#include <cctype>
#include <cfloat>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "nsfsi.h"

namespace {

struct Val {
  enum Kind { INT, FLT, BOOL, STR, LIST, GROUP } kind = INT;
  long long i = 0;
  double f = 0;
  bool b = false;
  std::string s;
  std::vector<Val> items;                     // LIST
  std::vector<std::pair<std::string, Val>> kv;  // GROUP
  const Val* find(const std::string& k) const {
    for (auto& p : kv)
      if (p.first == k) return &p.second;
    return nullptr;
  }
};

struct ConfigError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

class Reader {
 public:
  explicit Reader(const std::string& t) : t_(t) {}
  Val document() {
    Val root;
    root.kind = Val::GROUP;
    members(root, '\0');
    return root;
  }

 private:
  const std::string& t_;
  size_t p_ = 0;
  int line_ = 1;

  [[noreturn]] void bad(const std::string& m) {
    throw ConfigError("Parse error in ConfigFile, line " + std::to_string(line_) + ": " + m);
  }
  void ws() {
    while (p_ < t_.size()) {
      char c = t_[p_];
      if (c == '\n') {
        ++line_;
        ++p_;
      } else if (std::isspace(static_cast<unsigned char>(c))) {
        ++p_;
      } else if (c == '#' || t_.compare(p_, 2, "//") == 0) {
        while (p_ < t_.size() && t_[p_] != '\n') ++p_;
      } else if (t_.compare(p_, 2, "/*") == 0) {
        size_t e = t_.find("*/", p_ + 2);
        if (e == std::string::npos) bad("unterminated comment");
        for (size_t q = p_; q < e; ++q) line_ += t_[q] == '\n';
        p_ = e + 2;
      } else {
        break;
      }
    }
  }
  bool at(char c) {
    ws();
    return p_ < t_.size() && t_[p_] == c;
  }
  void members(Val& g, char close) {
    for (;;) {
      ws();
      if (p_ >= t_.size()) {
        if (close) bad("missing closing brace");
        return;
      }
      if (close && t_[p_] == close) {
        ++p_;
        return;
      }
      size_t b = p_;
      while (p_ < t_.size() && (std::isalnum(static_cast<unsigned char>(t_[p_])) || t_[p_] == '_' || t_[p_] == '-' ||
                                t_[p_] == '*'))
        ++p_;
      if (b == p_) bad("expected a setting name");
      std::string name = t_.substr(b, p_ - b);
      ws();
      if (p_ < t_.size() && (t_[p_] == '=' || t_[p_] == ':'))
        ++p_;
      else
        bad("expected '=' after '" + name + "'");
      g.kv.emplace_back(name, value());
      ws();
      if (p_ < t_.size() && (t_[p_] == ';' || t_[p_] == ',')) ++p_;
    }
  }
  Val value() {
    ws();
    if (p_ >= t_.size()) bad("missing value");
    Val v;
    char c = t_[p_];
    if (c == '{') {
      ++p_;
      v.kind = Val::GROUP;
      members(v, '}');
      return v;
    }
    if (c == '[' || c == '(') {
      char close = c == '[' ? ']' : ')';
      ++p_;
      v.kind = Val::LIST;
      if (at(close)) {
        ++p_;
        return v;
      }
      for (;;) {
        v.items.push_back(value());
        if (at(',')) {
          ++p_;
          continue;
        }
        if (at(close)) {
          ++p_;
          return v;
        }
        bad("expected ',' or closing bracket in list");
      }
    }
    if (c == '"') {
      v.kind = Val::STR;
      while (at('"')) {
        ++p_;
        while (p_ < t_.size() && t_[p_] != '"') {
          if (t_[p_] == '\\' && p_ + 1 < t_.size()) {
            ++p_;
            v.s += t_[p_] == 'n' ? '\n' : t_[p_] == 't' ? '\t' : t_[p_];
          } else {
            v.s += t_[p_];
          }
          ++p_;
        }
        if (p_ >= t_.size()) bad("unterminated string");
        ++p_;
      }
      return v;
    }
    size_t b = p_;
    while (p_ < t_.size() && (std::isalnum(static_cast<unsigned char>(t_[p_])) || std::strchr(".+-_", t_[p_]))) ++p_;
    std::string tok = t_.substr(b, p_ - b);
    std::string low;
    for (char ch : tok) low += static_cast<char>(std::tolower(static_cast<unsigned char>(ch)));
    if (low == "true" || low == "false") {
      v.kind = Val::BOOL;
      v.b = low == "true";
      return v;
    }
    bool hex = low.find("0x") != std::string::npos;
    char* end = nullptr;
    if (!hex && (low.find('.') != std::string::npos || low.find('e') != std::string::npos)) {
      v.kind = Val::FLT;
      v.f = std::strtod(tok.c_str(), &end);
    } else {
      v.kind = Val::INT;
      v.i = std::strtoll(tok.c_str(), &end, hex ? 16 : 10);
      while (end && (*end == 'L' || *end == 'l')) ++end;
    }
    if (tok.empty() || !end || *end) bad("bad value '" + tok + "'");
    return v;
  }
};

// Lookups with the reference's three failure classes (ConfigSettings.cpp:40-69).
const Val& need(const Val& g, const char* k) {
  const Val* v = g.find(k);
  if (!v) throw ConfigError(std::string("ConfigFile setting not found: ") + k);
  return *v;
}
long long asInt(const Val& v, const char* k) {
  if (v.kind != Val::INT) throw ConfigError(std::string("ConfigFile setting type mismatch: ") + k + " must be an integer");
  return v.i;
}
double asFlt(const Val& v, const char* k) {
  if (v.kind != Val::FLT)
    throw ConfigError(std::string("ConfigFile setting type mismatch: ") + k + " must be a float (with a decimal point)");
  return v.f;
}
bool asBool(const Val& v, const char* k) {
  if (v.kind != Val::BOOL) throw ConfigError(std::string("ConfigFile setting type mismatch: ") + k + " must be a boolean");
  return v.b;
}
std::string asStr(const Val& v, const char* k) {
  if (v.kind != Val::STR) throw ConfigError(std::string("ConfigFile setting type mismatch: ") + k + " must be a string");
  return v.s;
}
long long gi(const Val& g, const char* k) { return asInt(need(g, k), k); }
double gf(const Val& g, const char* k) { return asFlt(need(g, k), k); }
bool gb(const Val& g, const char* k) { return asBool(need(g, k), k); }
std::string gs(const Val& g, const char* k) { return asStr(need(g, k), k); }

int bcCode(const std::string& s) {
  if (s == "periodic") return NSF_BC_PERIODIC;
  if (s == "symmetry") return NSF_BC_SYMMETRY;
  if (s == "inlet") return NSF_BC_INLET;
  if (s == "outlet") return NSF_BC_OUTLET;
  throw ConfigError("case: unknown boundary type '" + s + "' (periodic, symmetry, inlet or outlet)");
}

void fill(const Val& root, nsf_config& c) {
  nsf_config_defaults(&c);
  c.NI = static_cast<unsigned>(gi(root, "NI"));
  c.NJ = static_cast<unsigned>(gi(root, "NJ"));
  c.NK = static_cast<unsigned>(gi(root, "NK"));
  std::string sc = gs(root, "stopCriterion");
  if (sc == "timesteps") {
    c.stop_criterion = 0;
    c.stop_time_level = static_cast<unsigned>(gi(root, "stopTimeLevel"));
  } else if (sc == "end_time") {
    c.stop_criterion = 1;
    c.t_end = gf(root, "t_end");
  } else {
    throw ConfigError("Error when reading ConfigFile. 'stopCriterion' needs to be 'timesteps' or 'end_time'.");
  }
  c.conv_stability_limit = gf(root, "convStabilityLimit");
  c.visc_stability_limit = gf(root, "viscStabilityLimit");
  const Val& fi = need(root, "filterIntervals");
  const Val& ft = need(root, "filterIntervalChangeTimes");
  if (fi.kind != Val::LIST || ft.kind != Val::LIST) throw ConfigError("filterIntervals and filterIntervalChangeTimes must be arrays");
  if (fi.items.size() > NSF_MAX_FILTER_INTERVALS || ft.items.size() > NSF_MAX_FILTER_INTERVALS)
    throw ConfigError("at most 16 filter intervals are supported");
  c.n_filter_intervals = static_cast<int>(fi.items.size());
  for (size_t q = 0; q < fi.items.size(); ++q)
    c.filter_intervals[q] = static_cast<unsigned>(asInt(fi.items[q], "filterIntervals"));
  c.n_filter_change_times = static_cast<int>(ft.items.size());
  for (size_t q = 0; q < ft.items.size(); ++q) c.filter_change_times[q] = asFlt(ft.items[q], "filterIntervalChangeTimes");
  // Same size rule as ConfigSettings.cpp:130-135 (size_t arithmetic: an empty interval list is an error).
  if (ft.items.size() > fi.items.size() || ft.items.size() < fi.items.size() - 1)
    throw ConfigError("filterIntervalChangeTimes must be the same size or one element smaller than filterIntervals.");
  c.status_report_interval = gf(root, "statusReportInterval");
  c.save_density = gb(root, "saveDensity");
  c.save_momentum = gb(root, "saveMomentum");
  c.save_energy = gb(root, "saveEnergy");
  c.save_velocity = gb(root, "saveVelocity");
  c.save_pressure = gb(root, "savePressure");
  c.save_temperature = gb(root, "saveTemperature");
  c.save_viscosity = gb(root, "saveViscosity");
  c.save_thermal_cond = gb(root, "saveThermalCond");
  c.save_ic = gb(root, "saveIC");
  c.save_final = gb(root, "saveFinal");
  c.save_intervals = gb(root, "saveIntervals");
  c.save_period = gf(root, "savePeriod");
  c.save_intervals_start_time = gf(root, "saveIntervalsStartTime");
  c.save_intervals_end_time = gf(root, "saveIntervalsEndTime");
  std::string ch = gs(root, "saveConvergenceHistory");
  if (ch == "none")
    c.conv_history = 0;
  else if (ch == "density")
    c.conv_history = 1;
  else if (ch == "all")
    c.conv_history = 2;
  else
    throw ConfigError("saveConvergenceHistory must be 'none', 'density' or 'all'.");
  c.gamma = gf(root, "Gamma");
  c.pr = gf(root, "Pr");
  c.r_gas = gf(root, "R");
  c.re = gf(root, "Re");
  if (root.find("sutherlands_C1")) c.sutherlands_c1 = gf(root, "sutherlands_C1");
  c.sutherlands_c2 = gf(root, "sutherlands_C2");
  c.m0 = gf(root, "M_0");
  c.t0 = gf(root, "T_0");
  c.lx = gf(root, "L_x");
  c.ly = gf(root, "L_y");
  c.lz = gf(root, "L_z");
  c.machine_precision_buffer = DBL_EPSILON * (c.lx + c.ly + c.lz);

  const Val* cs = root.find("case");
  if (!cs || gs(*cs, "kind") == "shipped") {
    c.shipped_case = 1;
    return;
  }
  if (gs(*cs, "kind") != "custom") throw ConfigError("case.kind must be 'shipped' or 'custom'");
  c.shipped_case = 0;
  const char* keys[3][2] = {{"bc_x_min", "bc_x_max"}, {"bc_y_min", "bc_y_max"}, {"bc_z_min", "bc_z_max"}};
  for (int a = 0; a < 3; ++a)
    for (int m = 0; m < 2; ++m) c.bc[a][m] = bcCode(gs(*cs, keys[a][m]));
  c.n_spheres = 0;
  if (const Val* sp = cs->find("spheres")) {
    if (sp->items.size() > NSF_MAX_SPHERES) throw ConfigError("too many spheres");
    for (auto& s : sp->items) {
      if (s.items.size() != 4) throw ConfigError("a sphere is (cx, cy, cz, r)");
      c.spheres[c.n_spheres++] = {asFlt(s.items[0], "sphere"), asFlt(s.items[1], "sphere"), asFlt(s.items[2], "sphere"),
                                  asFlt(s.items[3], "sphere")};
    }
  }
  c.n_cylinders = 0;
  if (const Val* cy = cs->find("cylinders")) {
    if (cy->items.size() > NSF_MAX_CYLINDERS) throw ConfigError("too many cylinders");
    for (auto& s : cy->items) {
      if (s.items.size() != 5) throw ConfigError("a cylinder is (axis, cx, cy, cz, r)");
      std::string ax = asStr(s.items[0], "cylinder axis");
      if (ax != "x" && ax != "y" && ax != "z") throw ConfigError("cylinder axis must be \"x\", \"y\" or \"z\"");
      c.cylinders[c.n_cylinders++] = {ax == "x" ? 0 : ax == "y" ? 1 : 2, asFlt(s.items[1], "cylinder"),
                                      asFlt(s.items[2], "cylinder"), asFlt(s.items[3], "cylinder"),
                                      asFlt(s.items[4], "cylinder")};
    }
  }
  std::string ic = gs(*cs, "ic");
  if (ic == "stagnation")
    c.ic = NSF_IC_STAGNATION;
  else if (ic == "freestream_noise")
    c.ic = NSF_IC_FREESTREAM_NOISE;
  else if (ic == "tgv")
    c.ic = NSF_IC_TGV;
  else
    throw ConfigError("case.ic must be 'stagnation', 'freestream_noise' or 'tgv'");
  c.noise_amp = cs->find("noise_amp") ? gf(*cs, "noise_amp") : 0.0;
  c.seed = cs->find("seed") ? static_cast<uint64_t>(gi(*cs, "seed")) : 0;
}

void report(char* err, size_t n, const char* m) {
  if (err && n) std::snprintf(err, n, "%s", m);
}

}  // namespace

extern "C" {

int32_t nsf_abi_version(void) { return NSF_ABI_VERSION; }

nsf_status nsf_config_defaults(nsf_config* c) {
  if (!c) return NSF_ERR_ARG;
  std::memset(c, 0, sizeof(*c));
  // Values of the reference's shipped ConfigFile and its hard-coded case (Mesh.cpp:33-55).
  c->NI = 161;
  c->NJ = 83;
  c->NK = 3;
  c->stop_criterion = 1;
  c->stop_time_level = 20;
  c->t_end = 200.;
  c->conv_stability_limit = 0.9;
  c->visc_stability_limit = -0.68;
  c->n_filter_intervals = 3;
  c->filter_intervals[0] = 50;
  c->filter_intervals[1] = 200;
  c->filter_intervals[2] = 1000;
  c->n_filter_change_times = 3;
  c->filter_change_times[0] = 30.;
  c->filter_change_times[1] = 60.;
  c->filter_change_times[2] = 100.;
  c->status_report_interval = 2.;
  c->save_density = c->save_velocity = c->save_pressure = c->save_temperature = 1;
  c->save_intervals = 1;
  c->save_period = 5.;
  c->conv_history = 2;
  c->gamma = 1.4;
  c->pr = 0.72;
  c->r_gas = 287.;
  c->re = 400.;
  c->sutherlands_c1 = 1.458e-6;
  c->sutherlands_c2 = 110.4;
  c->m0 = 0.25;
  c->t0 = 300.;
  c->lx = 2.;
  c->ly = 1.;
  c->lz = 0.05;
  c->machine_precision_buffer = DBL_EPSILON * (c->lx + c->ly + c->lz);
  c->shipped_case = 1;
  c->bc[0][0] = NSF_BC_INLET;
  c->bc[0][1] = NSF_BC_OUTLET;
  c->bc[1][0] = c->bc[1][1] = NSF_BC_SYMMETRY;
  c->bc[2][0] = c->bc[2][1] = NSF_BC_PERIODIC;
  c->ic = NSF_IC_STAGNATION;
  return NSF_OK;
}

nsf_status nsf_config_parse(const char* text, nsf_config* cfg, char* err, size_t errlen) {
  if (!text || !cfg) return NSF_ERR_ARG;
  try {
    std::string t(text);
    Reader r(t);
    Val root = r.document();
    nsf_config c;
    fill(root, c);
    *cfg = c;
    return NSF_OK;
  } catch (const std::exception& e) {
    report(err, errlen, e.what());
    return NSF_ERR_CONFIG;
  }
}

nsf_status nsf_config_load(const char* path, nsf_config* cfg, char* err, size_t errlen) {
  if (!path || !cfg) return NSF_ERR_ARG;
  std::ifstream in(path);
  if (!in) {
    std::string m = std::string("File I/O error: cannot open ") + path +
                    ". Make sure the 'ConfigFile' exists in correct path.";
    report(err, errlen, m.c_str());
    return NSF_ERR_CONFIG;
  }
  std::stringstream ss;
  ss << in.rdbuf();
  std::string text = ss.str();
  return nsf_config_parse(text.c_str(), cfg, err, errlen);
}

}  // extern "C"
