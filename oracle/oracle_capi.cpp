// Oracle test infrastructure only: C entry points over the CPU restatement in nsf_oracle.hpp, loaded with
// ctypes by tests/ and by bench.py's CPU-baseline leg. Never used by the product.
//
// Config reading mirrors ConfigSettings::readSettingValues (src/ConfigSettings.cpp:77-155) and
// setDerivedParameters (:160-163), plus the `case` group the parity cases use (boundary type per face,
// bodies, initial condition, seed). Parsing uses the oracle's libconfig stand-in (oracle/shim).
#include <chrono>
#include <cstdint>
#include <cstring>
#include <limits>
#include <string>

#include "libconfig.h++"
#include "nsf_dual.hpp"
#include "nsf_oracle.hpp"

using nsfo::Solver;

namespace {
struct Handle {
  Solver<double>* s = nullptr;
  double t = 0;
  unsigned long level = 0;
  std::string err;
  std::vector<double> dtHist, tHist;
};

int bcOf(const std::string& s) {
  if (s == "periodic") return nsfo::BC_PERIODIC;
  if (s == "symmetry") return nsfo::BC_SYMMETRY;
  if (s == "inlet") return nsfo::BC_INLET;
  if (s == "outlet") return nsfo::BC_OUTLET;
  throw std::runtime_error("unknown boundary type " + s);
}

void readParams(const libconfig::Config& cfg, nsfo::Params& P, nsfo::Case& C) {
  P.NI = (unsigned)cfg.lookup("NI");
  P.NJ = (unsigned)cfg.lookup("NJ");
  P.NK = (unsigned)cfg.lookup("NK");
  std::string sc = cfg.lookup("stopCriterion").c_str();
  if (sc == "timesteps") {
    P.stopEndTime = false;
    P.stopTimeLevel = (unsigned)cfg.lookup("stopTimeLevel");
  } else if (sc == "end_time") {
    P.stopEndTime = true;
    P.t_end = cfg.lookup("t_end");
  } else {
    throw std::runtime_error("stopCriterion");
  }
  P.convStabilityLimit = cfg.lookup("convStabilityLimit");
  P.viscStabilityLimit = cfg.lookup("viscStabilityLimit");
  const libconfig::Setting& fi = cfg.lookup("filterIntervals");
  for (int i = 0; i < fi.getLength(); ++i) P.filterIntervals.push_back((unsigned)fi[i]);
  const libconfig::Setting& ft = cfg.lookup("filterIntervalChangeTimes");
  for (int i = 0; i < ft.getLength(); ++i) P.filterIntervalChangeTimes.push_back(ft[i]);
  std::string ch = cfg.lookup("saveConvergenceHistory").c_str();
  P.convHistory = ch == "none" ? 0 : ch == "density" ? 1 : 2;
  P.Gamma = cfg.lookup("Gamma");
  P.Pr = cfg.lookup("Pr");
  P.Re = cfg.lookup("Re");
  P.sutherlands_C2 = cfg.lookup("sutherlands_C2");
  P.M_0 = cfg.lookup("M_0");
  P.T_0 = cfg.lookup("T_0");
  P.L_x = cfg.lookup("L_x");
  P.L_y = cfg.lookup("L_y");
  P.L_z = cfg.lookup("L_z");
  P.machinePrecisionBuffer = std::numeric_limits<double>::epsilon() * (P.L_x + P.L_y + P.L_z);
  if (!cfg.exists("case")) {
    C.shipped = true;
    return;
  }
  const libconfig::Setting& cs = cfg.lookup("case");
  std::string kind = cs["kind"].c_str();
  if (kind == "shipped") {
    C.shipped = true;
    return;
  }
  const char* keys[3][2] = {{"bc_x_min", "bc_x_max"}, {"bc_y_min", "bc_y_max"}, {"bc_z_min", "bc_z_max"}};
  for (int a = 0; a < 3; ++a)
    for (int m = 0; m < 2; ++m) C.bc[a][m] = bcOf(cs[keys[a][m]].c_str());
  if (cs.exists("spheres")) {
    const libconfig::Setting& sp = cs["spheres"];
    for (int b = 0; b < sp.getLength(); ++b)
      C.spheres.push_back({double(sp[b][0]), double(sp[b][1]), double(sp[b][2]), double(sp[b][3])});
  }
  if (cs.exists("cylinders")) {
    const libconfig::Setting& cy = cs["cylinders"];
    for (int b = 0; b < cy.getLength(); ++b) {
      std::string ax = cy[b][0].c_str();
      C.cylinders.push_back(
          {ax == "x" ? 0 : ax == "y" ? 1 : 2, double(cy[b][1]), double(cy[b][2]), double(cy[b][3]), double(cy[b][4])});
    }
  }
  std::string ic = cs["ic"].c_str();
  C.ic = ic == "stagnation" ? nsfo::IC_STAGNATION : ic == "freestream_noise" ? nsfo::IC_FREESTREAM_NOISE
         : ic == "tgv"      ? nsfo::IC_TGV
                            : -1;
  if (C.ic < 0) throw std::runtime_error("unknown ic " + ic);
  if (cs.exists("noise_amp")) C.noiseAmp = cs["noise_amp"];
  if (cs.exists("seed")) C.seed = static_cast<uint64_t>(static_cast<long long>(cs["seed"]));
}
}  // namespace

extern "C" {

void* nsfo_create(const char* cfgPath, int fromString, char* err, int errlen) {
  try {
    libconfig::Config cfg;
    if (fromString)
      cfg.readString(cfgPath);
    else
      cfg.readFile(cfgPath);
    nsfo::Params P;
    nsfo::Case C;
    readParams(cfg, P, C);
    auto* h = new Handle;
    h->s = new Solver<double>(P, C);
    return h;
  } catch (const std::exception& e) {
    if (err && errlen > 0) std::snprintf(err, errlen, "%s", e.what());
    return nullptr;
  }
}

int nsfo_initialize(void* hp, char* err, int errlen) {
  auto* h = static_cast<Handle*>(hp);
  try {
    h->s->initialize();
    return 0;
  } catch (const std::exception& e) {
    if (err && errlen > 0) std::snprintf(err, errlen, "%s", e.what());
    return 1;
  }
}

void nsfo_set_exact_image_solve(void* hp, int on) { static_cast<Handle*>(hp)->s->exactImageSolve = on != 0; }

void nsfo_set_frozen_dt(void* hp, const double* dts, uint64_t n) {
  auto* h = static_cast<Handle*>(hp);
  h->s->frozenDt.assign(dts, dts + n);
  h->s->dt = h->s->frozenDt[std::min<size_t>(h->s->stepCounter, n - 1)];
}

// Runs nsteps calls of marchTimeStep; returns wall seconds spent in the loop, or -1 if a step threw (the
// reference's own exceptions, e.g. a solid node around an image point, Boundary.cpp:723-724; the message is
// kept for nsfo_last_error).
double nsfo_march(void* hp, uint64_t nsteps) {
  auto* h = static_cast<Handle*>(hp);
  auto t0 = std::chrono::steady_clock::now();
  try {
    for (uint64_t s = 0; s < nsteps; ++s) {
      h->dtHist.push_back(h->s->dt);
      h->s->marchTimeStep(h->t, h->level);
      h->tHist.push_back(h->t);
    }
  } catch (const std::exception& e) {
    h->err = e.what();
    return -1.0;
  }
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// The message of the last failed call (empty if none); returns its length.
int nsfo_last_error(void* hp, char* buf, int len) {
  const std::string& e = static_cast<Handle*>(hp)->err;
  if (buf && len > 0) std::snprintf(buf, len, "%s", e.c_str());
  return int(e.size());
}

uint64_t nsfo_num_nodes(void* hp) { return static_cast<Handle*>(hp)->s->N; }
double nsfo_time(void* hp) { return static_cast<Handle*>(hp)->t; }
uint64_t nsfo_time_level(void* hp) { return static_cast<Handle*>(hp)->level; }
double nsfo_dt(void* hp) { return static_cast<Handle*>(hp)->s->dt; }
int nsfo_non_finite(void* hp) { return static_cast<Handle*>(hp)->s->nonFinite ? 1 : 0; }

void nsfo_geometry(void* hp, double* out6) {
  auto* s = static_cast<Handle*>(hp)->s;
  out6[0] = s->dx;
  out6[1] = s->dy;
  out6[2] = s->dz;
  out6[3] = s->off.x;
  out6[4] = s->off.y;
  out6[5] = s->off.z;
}

// 12 fields x N: rho, rho_u, rho_v, rho_w, rho_E, u, v, w, p, T, mu, kappa (current buffers).
void nsfo_get_fields(void* hp, double* out) {
  auto* s = static_cast<Handle*>(hp)->s;
  const std::vector<double>* a[12] = {&s->cons[0], &s->cons[1], &s->cons[2], &s->cons[3], &s->cons[4], &s->prim[0],
                                      &s->prim[1], &s->prim[2], &s->prim[3], &s->prim[4], &s->mu, &s->kappa};
  for (int f = 0; f < 12; ++f) std::memcpy(out + f * s->N, a[f]->data(), s->N * sizeof(double));
}
// The right-hand side (Solver.cpp:181-418) of the current conserved and stored primitive fields at the
// interior nodes (5 x N, zero elsewhere): a check of the RHS term table of the adjoint generator.
void nsfo_rhs(void* hp, double* out) {
  auto* s = static_cast<Handle*>(hp)->s;
  std::vector<double> k[5];
  for (auto& v : k) v.assign(s->N, 0.0);
  s->rhs(s->cons, k);
  for (int f = 0; f < 5; ++f) std::memcpy(out + f * s->N, k[f].data(), s->N * sizeof(double));
}

// The "old" conserved buffers (5 x N), which hold state the reference carries across steps.
void nsfo_get_old(void* hp, double* out) {
  auto* s = static_cast<Handle*>(hp)->s;
  for (int f = 0; f < 5; ++f) std::memcpy(out + f * s->N, s->old[f].data(), s->N * sizeof(double));
}
void nsfo_set_conserved(void* hp, const double* in5N) {
  auto* s = static_cast<Handle*>(hp)->s;
  for (int f = 0; f < 5; ++f) std::memcpy(s->cons[f].data(), in5N + f * s->N, s->N * sizeof(double));
}

void nsfo_get_types(void* hp, uint8_t* out) {
  auto* s = static_cast<Handle*>(hp)->s;
  std::memcpy(out, s->type.data(), s->N);
}
uint64_t nsfo_num_bodies(void* hp) { return static_cast<Handle*>(hp)->s->bodies.size(); }
uint64_t nsfo_num_ghosts(void* hp, uint64_t b) { return static_cast<Handle*>(hp)->s->bodies[b].ghosts.size(); }
uint64_t nsfo_num_filter(void* hp, uint64_t b) { return static_cast<Handle*>(hp)->s->bodies[b].filter.size(); }
uint64_t nsfo_closure_added(void* hp, uint64_t b) { return static_cast<Handle*>(hp)->s->bodies[b].closureAdded; }
// Per ghost: i, j, k as doubles, then body-intercept xyz, image-point xyz (9 doubles).
void nsfo_get_ghosts(void* hp, uint64_t b, double* out) {
  auto& g = static_cast<Handle*>(hp)->s->bodies[b].ghosts;
  for (size_t q = 0; q < g.size(); ++q) {
    double* o = out + 9 * q;
    o[0] = double(g[q].i);
    o[1] = double(g[q].j);
    o[2] = double(g[q].k);
    o[3] = g[q].bi.x;
    o[4] = g[q].bi.y;
    o[5] = g[q].bi.z;
    o[6] = g[q].ip.x;
    o[7] = g[q].ip.y;
    o[8] = g[q].ip.z;
  }
}
void nsfo_get_filter(void* hp, uint64_t b, uint64_t* out) {
  auto& f = static_cast<Handle*>(hp)->s->bodies[b].filter;
  for (size_t q = 0; q < f.size(); ++q) out[q] = f[q];
}
// History rows: t after step, dt used, 5 norms (-1 where not recorded).
uint64_t nsfo_history(void* hp, double* out) {
  auto* h = static_cast<Handle*>(hp);
  size_t n = h->dtHist.size();
  if (out)
    for (size_t s = 0; s < n; ++s) {
      out[7 * s + 0] = h->tHist[s];
      out[7 * s + 1] = h->dtHist[s];
      for (int f = 0; f < 5; ++f)
        out[7 * s + 2 + f] = s < h->s->normHist[f].size() ? h->s->normHist[f][s] : -1.0;
    }
  return n;
}

void nsfo_destroy(void* hp) {
  auto* h = static_cast<Handle*>(hp);
  delete h->s;
  delete h;
}

// The adjoint's objective and its directional derivative by forward-mode (dual-number) differentiation of
// a whole run: J = (1/navg) sum over the last navg of nsteps steps of the bodies' x-force (forceX), from
// the level-0 conserved field u0 + eps du0 (5 x N, every node; NULL u0: the case's initial condition) and
// the x-inlet profile factor inflow + eps dinflow (NJ x NK; NULL inflow: 1), with the dt sequence dts
// (nsteps values) frozen. NULL du0 / dinflow: no derivative along that parameter. Returns 0, or 1 with
// the message in err.
int nsfo_dual_objective(const char* cfgText, const double* u0, const double* du0, const double* inflow,
                        const double* dinflow, const double* dts, uint64_t nsteps, uint64_t navg, double* J,
                        double* dJ, char* err, int errlen) {
  using nsfo::Dual;
  try {
    libconfig::Config cfg;
    cfg.readString(cfgText);
    nsfo::Params P;
    nsfo::Case C;
    readParams(cfg, P, C);
    Solver<Dual> s(P, C);
    s.initialize();
    const size_t N = s.N;
    if (u0) {
      std::vector<Dual> U[5];
      for (int f = 0; f < 5; ++f) {
        U[f].resize(N);
        for (size_t q = 0; q < N; ++q) U[f][q] = Dual(u0[f * N + q], du0 ? du0[f * N + q] : 0.0);
      }
      s.setInitialConserved(U);
    }
    if (inflow) {
      s.inflowProfile.resize(s.NJ * s.NK);
      for (size_t q = 0; q < s.NJ * s.NK; ++q) s.inflowProfile[q] = Dual(inflow[q], dinflow ? dinflow[q] : 0.0);
    }
    s.frozenDt.assign(dts, dts + nsteps);
    s.dt = Dual(s.frozenDt[0]);
    double t = 0;
    unsigned long level = 0;
    Dual acc(0.0);
    for (uint64_t n = 0; n < nsteps; ++n) {
      s.marchTimeStep(t, level);
      if (n + 1 > nsteps - navg) acc += s.forceX() * (1.0 / double(navg));
    }
    *J = acc.v;
    *dJ = acc.d;
    return 0;
  } catch (const std::exception& e) {
    if (err && errlen > 0) std::snprintf(err, errlen, "%s", e.what());
    return 1;
  }
}
}
