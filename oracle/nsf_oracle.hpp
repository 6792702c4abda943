// Oracle test infrastructure only: never linked into, called by, or shipped with the product.
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may use it, as the checker.
//
// A CPU restatement of the reference solver's time-marching path (Frederik-Kris/3D-NS-FSI), written from
// its algorithm with the same loop order and floating-point expression order, so that built with
// -O3 -ffp-contract=off it reproduces the reference bit for bit (checked against oracle/_ref builds of the
// reference itself by tests/test_oracle_golden.py). Templated on the field scalar T so that the same code
// runs with dual numbers (forward-mode derivatives) for gradient checks. Geometry stays in double.
// Citations are path:line within the reference project.
#ifndef NSF_ORACLE_HPP
#define NSF_ORACLE_HPP

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <limits>
#include <map>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "fullpiv_lu.h"

namespace nsfo {

// NodeTypeEnum, src/Node.h:27-34 (same numeric values).
enum NodeType : uint8_t { FluidInterior = 0, FluidEdge = 1, FluidGhost = 2, SolidInactive = 3, SolidGhost = 4 };
enum BcType { BC_PERIODIC = 0, BC_SYMMETRY = 1, BC_INLET = 2, BC_OUTLET = 3 };
enum IcKind { IC_STAGNATION = 0, IC_FREESTREAM_NOISE = 1, IC_TGV = 2 };

// ConfigSettings public members, src/ConfigSettings.h:33-80 (those the time-marching path reads).
struct Params {
  size_t NI = 0, NJ = 0, NK = 0;
  bool stopEndTime = false;  // StopCriterionEnum::end_time
  unsigned long stopTimeLevel = 0;
  double t_end = 0;
  double convStabilityLimit = 0.5, viscStabilityLimit = -0.68;
  std::vector<unsigned> filterIntervals;
  std::vector<double> filterIntervalChangeTimes;
  int convHistory = 2;  // 0 none, 1 density, 2 all (ConvHistoryEnum)
  double Gamma = 1.4, Pr = 0.72, Re = 400, sutherlands_C2 = 110.4, M_0 = 0.25, T_0 = 300;
  double L_x = 1, L_y = 1, L_z = 1;
  double machinePrecisionBuffer = 0;  // ConfigSettings.cpp:160-163
};

struct Sphere {
  double cx, cy, cz, r;
};
struct Cylinder {
  int axis;
  double cx, cy, cz, r;
};
// The case description that the reference hard-codes in Mesh::setupBoundaries (Mesh.cpp:25-58) and
// Solver::applyStagnation_IC (Solver.cpp:31-51).
struct Case {
  bool shipped = false;  // the reference's own hard-coded case
  int bc[3][2] = {{BC_INLET, BC_OUTLET}, {BC_PERIODIC, BC_PERIODIC}, {BC_PERIODIC, BC_PERIODIC}};
  std::vector<Sphere> spheres;
  std::vector<Cylinder> cylinders;
  int ic = IC_STAGNATION;
  double noiseAmp = 0;
  uint64_t seed = 0;
};

// splitmix64 (Steele, Lea, Flood 2014); noise in [-1, 1). Shared definition of the seeded inputs.
inline uint64_t splitmix64(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ULL);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}
inline double noise_pm1(uint64_t& s) { return 2.0 * (static_cast<double>(splitmix64(s) >> 11) * 0x1.0p-53) - 1.0; }

struct V3 {  // Vector3_d, src/SmallVectors.h:15-25
  double x, y, z;
  double length() const { return std::sqrt(std::pow(x, 2) + std::pow(y, 2) + std::pow(z, 2)); }
  V3 operator+(V3 o) const { return {x + o.x, y + o.y, z + o.z}; }
  V3 operator-(V3 o) const { return {x - o.x, y - o.y, z - o.z}; }
  V3 operator*(double f) const { return {x * f, y * f, z * f}; }
  V3 operator/(double f) const { return {x / f, y / f, z / f}; }
};
struct Box {  // IndexBoundingBox, src/SmallVectors.h:72-104
  size_t iMin, iMax, jMin, jMax, kMin, kMax;
};
struct Ghost {  // GhostNode, src/Node.h:15-22
  size_t i, j, k;
  V3 bi, ip;
};

template <class T>
inline T tmax(const T& a, const T& b) {
  return (a < b) ? b : a;
}

template <class T>
class Solver {
 public:
  Params P;
  Case C;
  size_t NI, NJ, NK, N;
  double dx = -1, dy = -1, dz = -1;
  V3 off{0, 0, 0};
  // Fields (src/Mesh.h:82-86). cons[0..4] = rho, rho_u, rho_v, rho_w, rho_E; prim = u, v, w, p, T.
  std::vector<T> cons[5], old[5], prim[5], mu, kappa, k[4][5];
  std::vector<uint8_t> type;
  std::vector<size_t> interior, solidGhost;
  struct Edge {
    int axis, side, bc;
    Box owned;
  };
  std::vector<Edge> edges;  // application order (reversed claim order)
  struct Body {
    bool sphere;
    Sphere s;
    Cylinder c;
    std::vector<Ghost> ghosts;
    std::map<size_t, size_t> ghostMap;
    std::vector<size_t> filter;
    size_t closureAdded = 0;
  };
  std::vector<Body> bodies;
  T dt = T(0.0);
  std::vector<double> normHist[5];
  bool nonFinite = false;
  // Optional frozen dt sequence (used by gradient checks, where dt must not depend on the state).
  std::vector<double> frozenDt;
  // Optional: solve the image-point Vandermonde systems in extended precision (long double) instead of the
  // reference's double-precision complete-pivoting LU. The raw-coordinate matrices are ill-conditioned on
  // fine grids, so the reference's double solve amplifies last-bit differences of its inputs (up to ~1e-9
  // relative after two steps on a 1/126 grid); this mode gives the reference's algorithm with that rounding
  // amplification removed, as the comparison point for implementations that round differently.
  bool exactImageSolve = false;
  size_t stepCounter = 0;
  // Optional x-inlet velocity profile factor, index j * NK + k (the inlet velocity is min(1, t/10) M_0 times
  // the factor; empty: 1, the reference's uniform inflow). A parameter of the adjoint's gradient checks.
  std::vector<T> inflowProfile;

  explicit Solver(const Params& p, const Case& c)
      : P(p), C(c), NI(p.NI), NJ(p.NJ), NK(p.NK), N(p.NI * p.NJ * p.NK) {
    // Mesh::Mesh, src/Mesh.cpp:10-21: every array is value-initialised (zero).
    for (int f = 0; f < 5; ++f) {
      cons[f].assign(N, T(0.0));
      old[f].assign(N, T(0.0));
      prim[f].assign(N, T(0.0));
      for (int s = 0; s < 4; ++s) k[s][f].assign(N, T(0.0));
    }
    mu.assign(N, T(0.0));
    kappa.assign(N, T(0.0));
    type.assign(N, FluidInterior);
  }

  size_t id(size_t i, size_t j, size_t kk) const { return i * NJ * NK + j * NK + kk; }  // SmallVectors.h:46-50
  void ijk(size_t idx, size_t& i, size_t& j, size_t& kk) const {                        // SmallVectors.h:37-43
    i = idx / (NJ * NK);
    j = idx % (NJ * NK) / NK;
    kk = idx % (NJ * NK) % NK;
  }
  V3 pos(size_t i, size_t j, size_t kk) const {  // getNodePosition, SmallVectors.h:56-64
    return {(static_cast<int>(i) - off.x) * dx, (static_cast<int>(j) - off.y) * dy, (static_cast<int>(kk) - off.z) * dz};
  }
  Box surrounding(const V3& p) const {  // getSurroundingNodesBox, SmallVectors.h:108-127
    size_t iN = static_cast<size_t>(std::ceil(p.x / dx) + off.x);
    size_t jN = static_cast<size_t>(std::ceil(p.y / dy) + off.y);
    size_t kN = static_cast<size_t>(std::ceil(p.z / dz) + off.z);
    iN = std::max<size_t>(iN, 1);
    jN = std::max<size_t>(jN, 1);
    kN = std::max<size_t>(kN, 1);
    iN = std::min<size_t>(iN, NI);
    jN = std::min<size_t>(jN, NJ);
    kN = std::min<size_t>(kN, NK);
    return {iN - 1, iN, jN - 1, jN, kN - 1, kN};
  }
  void corners(const Box& b, size_t out[8]) const {  // IndexBoundingBox::asIndexList, SmallVectors.h:89-103
    out[0] = id(b.iMin, b.jMin, b.kMin);
    out[1] = id(b.iMin, b.jMin, b.kMax);
    out[2] = id(b.iMin, b.jMax, b.kMin);
    out[3] = id(b.iMin, b.jMax, b.kMax);
    out[4] = id(b.iMax, b.jMin, b.kMin);
    out[5] = id(b.iMax, b.jMin, b.kMax);
    out[6] = id(b.iMax, b.jMax, b.kMin);
    out[7] = id(b.iMax, b.jMax, b.kMax);
  }

  // ---------------- thermodynamics, src/FlowVariableGroupStructs.h:152-186 ----------------
  void deriveConserved(const T pr[5], T cv[5]) const {
    const T &u = pr[0], &v = pr[1], &w = pr[2], &p = pr[3], &Tt = pr[4];
    T rho = (P.Gamma * p - Tt) / (1 + Tt);
    cv[0] = rho;
    cv[1] = (1 + rho) * u;
    cv[2] = (1 + rho) * v;
    cv[3] = (1 + rho) * w;
    cv[4] = p / (P.Gamma - 1) + (1 + rho) / 2 * (u * u + v * v + w * w);
  }
  void derivePrimitive(const T cv[5], T pr[5]) const {
    const T &rho = cv[0], &ru = cv[1], &rv = cv[2], &rw = cv[3], &rE = cv[4];
    T u = ru / (1 + rho), v = rv / (1 + rho), w = rw / (1 + rho);
    T p = (P.Gamma - 1) * (rE - (1 + rho) / 2 * (u * u + v * v + w * w));
    T Tt = (P.Gamma * p - rho) / (1 + rho);
    pr[0] = u;
    pr[1] = v;
    pr[2] = w;
    pr[3] = p;
    pr[4] = Tt;
  }
  void deriveTransport(const T pr[5], T& m, T& kap) const {
    const T& Tt = pr[4];
    double ScPlusOne = 1 + P.sutherlands_C2 / P.T_0;
    using std::pow;
    m = pow(1 + Tt, 1.5) * ScPlusOne / (P.Re * (Tt + ScPlusOne));
    kap = m / ((P.Gamma - 1) * P.Pr);
  }
  void setAll(size_t idx, const T cv[5], const T pr[5], const T& m, const T& kap) {  // :189-206
    for (int f = 0; f < 5; ++f) {
      cons[f][idx] = cv[f];
      prim[f][idx] = pr[f];
    }
    mu[idx] = m;
    kappa[idx] = kap;
  }

  // ---------------- setup ----------------
  // Mesh::setupBoundaries (Mesh.cpp:25-58) generalised to a case description: claim order z-min, z-max,
  // y-min, y-max, x-min, x-max; spacing/offset rules of Mesh.cpp:44-49.
  void setupBoundaries() {
    if (C.shipped) {
      C.bc[2][0] = C.bc[2][1] = BC_PERIODIC;
      C.bc[1][0] = C.bc[1][1] = BC_SYMMETRY;
      C.bc[0][0] = BC_INLET;
      C.bc[0][1] = BC_OUTLET;
      C.spheres.clear();
      C.cylinders = {Cylinder{2, P.L_x / 4, P.L_y / 2, 0, P.L_y / 10}};
      C.ic = IC_STAGNATION;
    }
    size_t n[3] = {NI, NJ, NK};
    double L[3] = {P.L_x, P.L_y, P.L_z};
    double d[3], o[3];
    for (int a = 0; a < 3; ++a) {
      int t = C.bc[a][0];
      if (t == BC_PERIODIC) {
        d[a] = L[a] / (n[a] - 2);
        o[a] = 1;
      } else if (t == BC_SYMMETRY) {
        d[a] = L[a] / (n[a] - 3);
        o[a] = 1;
      } else {
        d[a] = L[a] / (n[a] - 1);
        o[a] = 0;
      }
    }
    dx = d[0];
    dy = d[1];
    dz = d[2];
    off = {o[0], o[1], o[2]};
    for (auto& s : C.spheres) {
      Body b{};
      b.sphere = true;
      b.s = s;
      bodies.push_back(b);
    }
    for (auto& c : C.cylinders) {
      Body b{};
      b.sphere = false;
      b.c = c;
      bodies.push_back(b);
    }
  }

  // Mesh::categorizeNodes, Mesh.cpp:61-82 with MeshEdgeBoundary::identifyOwnedNodes, Boundary.cpp:18-71.
  void categorizeNodes() {
    std::fill(type.begin(), type.end(), FluidInterior);
    Box unclaimed{0, NI - 1, 0, NJ - 1, 0, NK - 1};
    std::vector<Edge> claimed;
    for (int a = 2; a >= 0; --a)
      for (int m = 0; m < 2; ++m) {
        Edge e{a, m, C.bc[a][m], unclaimed};
        if (a == 0) {
          if (m == 0) {
            e.owned.iMax = e.owned.iMin;
            unclaimed.iMin++;
          } else {
            e.owned.iMin = e.owned.iMax;
            unclaimed.iMax--;
          }
        } else if (a == 1) {
          if (m == 0) {
            e.owned.jMax = e.owned.jMin;
            unclaimed.jMin++;
          } else {
            e.owned.jMin = e.owned.jMax;
            unclaimed.jMax--;
          }
        } else {
          if (m == 0) {
            e.owned.kMax = e.owned.kMin;
            unclaimed.kMin++;
          } else {
            e.owned.kMin = e.owned.kMax;
            unclaimed.kMax--;
          }
        }
        uint8_t t = (e.bc == BC_INLET || e.bc == BC_OUTLET) ? FluidEdge : FluidGhost;
        for (size_t i = e.owned.iMin; i <= e.owned.iMax; ++i)
          for (size_t j = e.owned.jMin; j <= e.owned.jMax; ++j)
            for (size_t kk = e.owned.kMin; kk <= e.owned.kMax; ++kk) type[id(i, j, kk)] = t;
        claimed.push_back(e);
      }
    edges.assign(claimed.rbegin(), claimed.rend());
    for (auto& b : bodies) identifyRelatedNodes(b);
    interior.clear();
    solidGhost.clear();
    for (size_t idx = 0; idx < N; ++idx)
      if (type[idx] == FluidInterior)
        interior.push_back(idx);
      else if (type[idx] == SolidGhost)
        solidGhost.push_back(idx);
  }

  V3 normalProbe(const Body& b, const V3& g) const {  // Boundary.cpp:920-935 (cylinder), :1047-1053 (sphere)
    V3 c2g;
    double r;
    if (b.sphere) {
      c2g = g - V3{b.s.cx, b.s.cy, b.s.cz};
      r = b.s.r;
    } else {
      c2g = g - V3{b.c.cx, b.c.cy, b.c.cz};
      if (b.c.axis == 0) c2g.x = 0;
      if (b.c.axis == 1) c2g.y = 0;
      if (b.c.axis == 2) c2g.z = 0;
      r = b.c.r;
    }
    double lengthFactor = (r - c2g.length()) / c2g.length();
    return c2g * lengthFactor;
  }

  // {Sphere,Cylinder}Body::identifyRelatedNodes: Boundary.cpp:894-917 and :1023-1044, with the bounding
  // boxes of :938-965 / :1056-1072, the solid/filter scans of :968-1014 / :1075-1103, the 18-neighbour ghost
  // test of :461-562 and the image-point closure of :582-615 (the well-defined cylinder form of the loop).
  void identifyRelatedNodes(Body& b) {
    const size_t layer = 2;
    Box box;
    if (b.sphere) {
      size_t rX = static_cast<size_t>(std::ceil(b.s.r / dx)) + 1 + layer;
      size_t rY = static_cast<size_t>(std::ceil(b.s.r / dy)) + 1 + layer;
      size_t rZ = static_cast<size_t>(std::ceil(b.s.r / dz)) + 1 + layer;
      size_t cX = static_cast<size_t>(std::round(b.s.cx / dx));
      size_t cY = static_cast<size_t>(std::round(b.s.cy / dy));
      size_t cZ = static_cast<size_t>(std::round(b.s.cz / dz));
      box = {cX - rX, cX + rX, cY - rY, cY + rY, cZ - rZ, cZ + rZ};
    } else {
      size_t rX = static_cast<size_t>(std::ceil(b.c.r / dx)) + 1 + layer;
      size_t rY = static_cast<size_t>(std::ceil(b.c.r / dy)) + 1 + layer;
      size_t rZ = static_cast<size_t>(std::ceil(b.c.r / dz)) + 1 + layer;
      size_t cX = static_cast<size_t>(std::round(b.c.cx / dx));
      size_t cY = static_cast<size_t>(std::round(b.c.cy / dy));
      size_t cZ = static_cast<size_t>(std::round(b.c.cz / dz));
      box = {0, NI - 1, 0, NJ - 1, 0, NK - 1};
      if (b.c.axis != 0) {
        box.iMin = cX - rX;
        box.iMax = cX + rX;
      }
      if (b.c.axis != 1) {
        box.jMin = cY - rY;
        box.jMax = cY + rY;
      }
      if (b.c.axis != 2) {
        box.kMin = cZ - rZ;
        box.kMax = cZ + rZ;
      }
    }
    if (box.iMin > box.iMax || box.iMax >= NI || box.jMin > box.jMax || box.jMax >= NJ || box.kMin > box.kMax ||
        box.kMax >= NK)
      throw std::runtime_error("body bounding box leaves the mesh (the reference does not clamp it)");
    std::vector<size_t> solids;
    double filterWidthSphere = layer * std::max({dx, dy, dz});
    for (size_t i = box.iMin; i <= box.iMax; ++i)
      for (size_t j = box.jMin; j <= box.jMax; ++j)
        for (size_t kk = box.kMin; kk <= box.kMax; ++kk) {
          V3 p = pos(i, j, kk);
          double dist, r, fw;
          if (b.sphere) {
            dist = std::sqrt(std::pow(p.x - b.s.cx, 2) + std::pow(p.y - b.s.cy, 2) + std::pow(p.z - b.s.cz, 2));
            r = b.s.r;
            fw = filterWidthSphere;
          } else {
            r = b.c.r;
            if (b.c.axis == 0) {
              dist = std::sqrt(std::pow(p.y - b.c.cy, 2) + std::pow(p.z - b.c.cz, 2));
              fw = layer * std::max(dy, dz);
            } else if (b.c.axis == 1) {
              dist = std::sqrt(std::pow(p.x - b.c.cx, 2) + std::pow(p.z - b.c.cz, 2));
              fw = layer * std::max(dx, dz);
            } else {
              dist = std::sqrt(std::pow(p.x - b.c.cx, 2) + std::pow(p.y - b.c.cy, 2));
              fw = layer * std::max(dx, dy);
            }
          }
          if (dist < r - P.machinePrecisionBuffer) {
            type[id(i, j, kk)] = SolidInactive;
            solids.push_back(id(i, j, kk));
          } else if (dist < r + fw && type[id(i, j, kk)] == FluidInterior)
            b.filter.push_back(id(i, j, kk));
        }
    // findGhostNodesWithFluidNeighbors, Boundary.cpp:461-562
    for (size_t idx : solids) {
      size_t i, j, kk;
      ijk(idx, i, j, kk);
      bool has = false;
      auto fi = [&](size_t a, size_t bb, size_t c) {
        if (type[id(a, bb, c)] == FluidInterior) has = true;
      };
      if (i > 0) {
        fi(i - 1, j, kk);
        if (j > 0) fi(i - 1, j - 1, kk);
        if (j < NJ - 1) fi(i - 1, j + 1, kk);
        if (kk > 0) fi(i - 1, j, kk - 1);
        if (kk < NK - 1) fi(i - 1, j, kk + 1);
      }
      if (i < NI - 1) {
        fi(i + 1, j, kk);
        if (j > 0) fi(i + 1, j - 1, kk);
        if (j < NJ - 1) fi(i + 1, j + 1, kk);
        if (kk > 0) fi(i + 1, j, kk - 1);
        if (kk < NK - 1) fi(i + 1, j, kk + 1);
      }
      if (j > 0) {
        fi(i, j - 1, kk);
        if (kk > 0) fi(i, j - 1, kk - 1);
        if (kk < NK - 1) fi(i, j - 1, kk + 1);
      }
      if (j < NJ - 1) {
        fi(i, j + 1, kk);
        if (kk > 0) fi(i, j + 1, kk - 1);
        if (kk < NK - 1) fi(i, j + 1, kk + 1);
      }
      if (kk > 0) fi(i, j, kk - 1);
      if (kk < NK - 1) fi(i, j, kk + 1);
      if (has) {
        b.ghostMap[idx] = b.ghosts.size();
        b.ghosts.push_back(Ghost{i, j, kk, {0, 0, 0}, {0, 0, 0}});
        type[idx] = SolidGhost;
      }
    }
    size_t first = 0;
    for (;;) {
      std::vector<Ghost> fresh;
      for (size_t g = first; g < b.ghosts.size(); ++g) {
        Ghost& gh = b.ghosts[g];
        V3 gp = pos(gh.i, gh.j, gh.k);
        V3 np = normalProbe(b, gp);
        gh.bi = gp + np;
        gh.ip = gh.bi + np;
        Box sb = surrounding(gh.ip);
        size_t cs[8];
        corners(sb, cs);
        for (size_t c : cs)
          if (type[c] == SolidInactive) {
            size_t a, bb, cc;
            ijk(c, a, bb, cc);
            fresh.push_back(Ghost{a, bb, cc, {0, 0, 0}, {0, 0, 0}});
            type[c] = SolidGhost;
          }
      }
      if (fresh.empty()) break;
      first = b.ghosts.size();
      for (auto& g : fresh) {
        b.ghostMap[id(g.i, g.j, g.k)] = b.ghosts.size();
        b.ghosts.push_back(g);
      }
      b.closureAdded += fresh.size();
    }
  }

  void applyInitialCondition() {
    const double M = P.M_0;
    uint64_t s = C.seed;
    for (size_t idx = 0; idx < N; ++idx) {
      double u = 0, v = 0, w = 0, p = 0, Tt = 0;
      if (C.ic == IC_FREESTREAM_NOISE) {
        u = M + C.noiseAmp * noise_pm1(s);
        v = C.noiseAmp * noise_pm1(s);
        w = C.noiseAmp * noise_pm1(s);
      } else if (C.ic == IC_TGV) {
        size_t i, j, kk;
        ijk(idx, i, j, kk);
        V3 X = pos(i, j, kk);
        u = M * std::sin(X.x) * std::cos(X.y) * std::cos(X.z);
        v = -M * std::cos(X.x) * std::sin(X.y) * std::cos(X.z);
        w = 0;
        p = M * M / 16 * (std::cos(2 * X.x) + std::cos(2 * X.y)) * (std::cos(2 * X.z) + 2);
      }
      T pr[5] = {T(u), T(v), T(w), T(p), T(Tt)}, cv[5], m, kap;
      deriveConserved(pr, cv);
      deriveTransport(pr, m, kap);
      setAll(idx, cv, pr, m, kap);
    }
  }

  // Solver::initialize, Solver.cpp:22-28.
  void initialize() {
    setupBoundaries();
    categorizeNodes();
    applyInitialCondition();
    updateTimeStepSize(0);
  }

  // ---------------- time step size, Solver.cpp:80-126 ----------------
  T inviscidLimit() const {
    T mX = T(0.0), mY = T(0.0), mZ = T(0.0);
    using std::fabs;
    using std::sqrt;
    for (size_t i = 0; i < N; ++i) {
      T c = sqrt((1 + P.Gamma * prim[3][i]) / (1 + cons[0][i]));
      mX = tmax(mX, c + fabs(prim[0][i]));
      mY = tmax(mY, c + fabs(prim[1][i]));
      mZ = tmax(mZ, c + fabs(prim[2][i]));
    }
    return std::fabs(P.convStabilityLimit) / (mX / dx + mY / dy + mZ / dz);
  }
  T viscousLimit() const {
    double mod = std::max(4. / 3, P.Gamma / P.Pr);
    T mNu = T(0.0);
    for (size_t i = 0; i < N; ++i) mNu = tmax(mNu, mu[i] / (cons[0][i] + 1) * mod);
    double dx2 = dx * dx, dy2 = dy * dy, dz2 = dz * dz;
    return std::fabs(P.viscStabilityLimit) / (mNu * (1 / dx2 + 1 / dy2 + 1 / dz2));
  }
  void updateTimeStepSize(double t) {
    if (!frozenDt.empty()) {
      dt = T(frozenDt[std::min(stepCounter, frozenDt.size() - 1)]);
      return;
    }
    T a = inviscidLimit(), b = viscousLimit();
    dt = (b < a) ? b : a;
    if (P.stopEndTime && t + dt > P.t_end) dt = T(P.t_end - t);
  }

  // ---------------- RHS, Solver.cpp:181-418 ----------------
  void rhs(std::vector<T>* U, std::vector<T>* out) {
    const std::vector<T>&ru = U[1], &rv = U[2], &rw = U[3], &E = U[4];
    const std::vector<T>&u = prim[0], &v = prim[1], &w = prim[2], &p = prim[3], &Tt = prim[4], &m = mu,
                         &kp = kappa;
    const size_t sI = NJ * NK, sJ = NK;
    // continuity, Solver.cpp:181-196
    for (size_t n : interior) {
      T fx = -(ru[n + sI] - ru[n - sI]) / (2 * dx);
      T fy = -(rv[n + sJ] - rv[n - sJ]) / (2 * dy);
      T fz = -(rw[n + 1] - rw[n - 1]) / (2 * dz);
      out[0][n] = fx + fy + fz;
    }
    // x-momentum, Solver.cpp:199-243
    {
      double a = -1. / (2 * dx), b = -1. / (2 * dy), c = -1. / (2 * dz), xx = 2. / (3 * dx * dx),
             yy = 1. / (2 * dy * dy), zz = 1. / (2 * dz * dz), yx = -1. / (6 * dy * dx), xy = 1. / (4 * dx * dy),
             zx = -1. / (6 * dz * dx), xz = 1. / (4 * dx * dz);
      for (size_t n : interior) {
        const size_t E_ = n + sI, W = n - sI, N_ = n + sJ, S = n - sJ, U_ = n + 1, D = n - 1;
        T cX = a * (ru[E_] * u[E_] + p[E_] - ru[W] * u[W] - p[W]);
        T cY = b * (ru[N_] * v[N_] - ru[S] * v[S]);
        T cZ = c * (ru[U_] * w[U_] - ru[D] * w[D]);
        T vXX = xx * ((m[E_] + m[n]) * (u[E_] - u[n]) - (m[W] + m[n]) * (u[n] - u[W]));
        T vYY = yy * ((m[N_] + m[n]) * (u[N_] - u[n]) - (m[S] + m[n]) * (u[n] - u[S]));
        T vZZ = zz * ((m[U_] + m[n]) * (u[U_] - u[n]) - (m[D] + m[n]) * (u[n] - u[D]));
        T vXY = xy * (m[N_] * (v[E_ + sJ] - v[W + sJ]) - m[S] * (v[E_ - sJ] - v[W - sJ]));
        T vYX = yx * (m[E_] * (v[E_ + sJ] - v[E_ - sJ]) - m[W] * (v[W + sJ] - v[W - sJ]));
        T vXZ = xz * (m[U_] * (w[E_ + 1] - w[W + 1]) - m[D] * (w[E_ - 1] - w[W - 1]));
        T vZX = zx * (m[E_] * (w[E_ + 1] - w[E_ - 1]) - m[W] * (w[W + 1] - w[W - 1]));
        out[1][n] = cX + cY + cZ + vXX + vYY + vZZ + vXY + vYX + vXZ + vZX;
      }
    }
    // y-momentum, Solver.cpp:246-290
    {
      double a = -1. / (2 * dx), b = -1. / (2 * dy), c = -1. / (2 * dz), xx = 1. / (2 * dx * dx),
             yy = 2. / (3 * dy * dy), zz = 1. / (2 * dz * dz), xy6 = -1. / (6 * dx * dy), yx4 = 1. / (4 * dy * dx),
             zy6 = -1. / (6 * dz * dy), yz4 = 1. / (4 * dy * dz);
      for (size_t n : interior) {
        const size_t E_ = n + sI, W = n - sI, N_ = n + sJ, S = n - sJ, U_ = n + 1, D = n - 1;
        T cX = a * (rv[E_] * u[E_] - rv[W] * u[W]);
        T cY = b * (rv[N_] * v[N_] + p[N_] - rv[S] * v[S] - p[S]);
        T cZ = c * (rv[U_] * w[U_] - rv[D] * w[D]);
        T vXX = xx * ((m[E_] + m[n]) * (v[E_] - v[n]) - (m[W] + m[n]) * (v[n] - v[W]));
        T vYY = yy * ((m[N_] + m[n]) * (v[N_] - v[n]) - (m[S] + m[n]) * (v[n] - v[S]));
        T vZZ = zz * ((m[U_] + m[n]) * (v[U_] - v[n]) - (m[D] + m[n]) * (v[n] - v[D]));
        T vYX = yx4 * (m[E_] * (u[E_ + sJ] - u[E_ - sJ]) - m[W] * (u[W + sJ] - u[W - sJ]));
        T vXY = xy6 * (m[N_] * (u[E_ + sJ] - u[W + sJ]) - m[S] * (u[E_ - sJ] - u[W - sJ]));
        T vYZ = yz4 * (m[U_] * (w[N_ + 1] - w[S + 1]) - m[D] * (w[N_ - 1] - w[S - 1]));
        T vZY = zy6 * (m[N_] * (w[N_ + 1] - w[N_ - 1]) - m[S] * (w[S + 1] - w[S - 1]));
        out[2][n] = cX + cY + cZ + vXX + vYY + vZZ + vYX + vXY + vYZ + vZY;
      }
    }
    // z-momentum, Solver.cpp:293-339
    {
      double a = -1. / (2 * dx), b = -1. / (2 * dy), c = -1. / (2 * dz), xx = 1. / (2 * dx * dx),
             yy = 1. / (2 * dy * dy), zz = 2. / (3 * dz * dz), zx4 = 1. / (4 * dz * dx), xz6 = -1. / (6 * dx * dz),
             zy4 = 1. / (4 * dz * dy), yz6 = -1. / (6 * dy * dz);
      for (size_t n : interior) {
        const size_t E_ = n + sI, W = n - sI, N_ = n + sJ, S = n - sJ, U_ = n + 1, D = n - 1;
        T cX = a * (rw[E_] * u[E_] - rw[W] * u[W]);
        T cY = b * (rw[N_] * v[N_] - rw[S] * v[S]);
        T cZ = c * (rw[U_] * w[U_] + p[U_] - rw[D] * w[D] - p[D]);
        T vXX = xx * ((m[E_] + m[n]) * (w[E_] - w[n]) - (m[W] + m[n]) * (w[n] - w[W]));
        T vYY = yy * ((m[N_] + m[n]) * (w[N_] - w[n]) - (m[S] + m[n]) * (w[n] - w[S]));
        T vZZ = zz * ((m[U_] + m[n]) * (w[U_] - w[n]) - (m[D] + m[n]) * (w[n] - w[D]));
        T vZX = zx4 * (m[E_] * (u[E_ + 1] - u[E_ - 1]) - m[W] * (u[W + 1] - u[W - 1]));
        T vXZ = xz6 * (m[U_] * (u[E_ + 1] - u[W + 1]) - m[D] * (u[E_ - 1] - u[W - 1]));
        T vZY = zy4 * (m[N_] * (v[N_ + 1] - v[N_ - 1]) - m[S] * (v[S + 1] - v[S - 1]));
        T vYZ = yz6 * (m[U_] * (v[N_ + 1] - v[S + 1]) - m[D] * (v[N_ - 1] - v[S - 1]));
        out[3][n] = cX + cY + cZ + vXX + vYY + vZZ + vZX + vXZ + vZY + vYZ;
      }
    }
    // energy, Solver.cpp:342-418
    {
      double a = -1. / (2 * dx), b = -1. / (2 * dy), c = -1. / (2 * dz), xx23 = 2. / (3 * dx * dx),
             xx12 = 1. / (2 * dx * dx), yx6 = -1. / (6 * dy * dx), zx6 = -1. / (6 * dz * dx), yx4 = 1. / (4 * dy * dx),
             zx4 = 1. / (4 * dz * dx), yy12 = 1. / (2 * dy * dy), yy23 = 2. / (3 * dy * dy), zy6 = -1. / (6 * dz * dy),
             zy4 = 1. / (4 * dz * dy), zz12 = 1. / (2 * dz * dz), zz23 = 2. / (3 * dz * dz);
      double H0 = 1. / (P.Gamma - 1);
      for (size_t n : interior) {
        const size_t E_ = n + sI, W = n - sI, N_ = n + sJ, S = n - sJ, U_ = n + 1, D = n - 1;
        const T mP = m[n], mW = m[W], mE = m[E_], mS = m[S], mN = m[N_], mD = m[D], mU = m[U_];
        const T uP = u[n], uW = u[W], uE = u[E_], uS = u[S], uN = u[N_], uD = u[D], uU = u[U_];
        const T vP = v[n], vW = v[W], vE = v[E_], vS = v[S], vN = v[N_], vD = v[D], vU = v[U_];
        const T wP = w[n], wW = w[W], wE = w[E_], wS = w[S], wN = w[N_], wD = w[D], wU = w[U_];
        const T kP = kp[n], TP = Tt[n];
        T inv = a * ((H0 + E[E_] + p[E_]) * uE - (H0 + E[W] + p[W]) * uW) +
                b * ((H0 + E[N_] + p[N_]) * vN - (H0 + E[S] + p[S]) * vS) +
                c * ((H0 + E[U_] + p[U_]) * wU - (H0 + E[D] + p[D]) * wD);
        T vfX = xx23 * ((mE * uE + mP * uP) * (uE - uP) - (mW * uW + mP * uP) * (uP - uW)) +
                xx12 * ((mE * vE + mP * vP) * (vE - vP) - (mW * vW + mP * vP) * (vP - vW)) +
                xx12 * ((mE * wE + mP * wP) * (wE - wP) - (mW * wW + mP * wP) * (wP - wW)) +
                yx6 * (mE * uE * (v[E_ + sJ] - v[E_ - sJ]) - mW * uW * (v[W + sJ] - v[W - sJ])) +
                zx6 * (mE * uE * (w[E_ + 1] - w[E_ - 1]) - mW * uW * (w[W + 1] - w[W - 1])) +
                yx4 * (mE * vE * (u[E_ + sJ] - u[E_ - sJ]) - mW * vW * (u[W + sJ] - u[W - sJ])) +
                zx4 * (mE * wE * (u[E_ + 1] - u[E_ - 1]) - mW * wW * (u[W + 1] - u[W - 1]));
        T vfY = yy12 * ((mN * uN + mP * uP) * (uN - uP) - (mS * uS + mP * uP) * (uP - uS)) +
                yy23 * ((mN * vN + mP * vP) * (vN - vP) - (mS * vS + mP * vP) * (vP - vS)) +
                yy12 * ((mN * wN + mP * wP) * (wN - wP) - (mS * wS + mP * wP) * (wP - wS)) +
                yx6 * (mN * vN * (u[E_ + sJ] - u[W + sJ]) - mS * vS * (u[E_ - sJ] - u[W - sJ])) +
                zy6 * (mN * vN * (w[N_ + 1] - w[N_ - 1]) - mS * vS * (w[S + 1] - w[S - 1])) +
                yx4 * (mN * uN * (v[E_ + sJ] - v[W + sJ]) - mS * uS * (v[E_ - sJ] - v[W - sJ])) +
                zy4 * (mN * wN * (v[N_ + 1] - v[N_ - 1]) - mS * wS * (v[S + 1] - v[S - 1]));
        T vfZ = zz12 * ((mU * uU + mP * uP) * (uU - uP) - (mD * uD + mP * uP) * (uP - uD)) +
                zz12 * ((mU * vU + mP * vP) * (vU - vP) - (mD * vD + mP * vP) * (vP - vD)) +
                zz23 * ((mU * wU + mP * wP) * (wU - wP) - (mD * wD + mP * wP) * (wP - wD)) +
                zx6 * (mU * wU * (u[E_ + 1] - u[W + 1]) - mD * wD * (u[E_ - 1] - u[W - 1])) +
                zy6 * (mU * wU * (v[N_ + 1] - v[S + 1]) - mD * wD * (v[N_ - 1] - v[S - 1])) +
                zx4 * (mU * uU * (w[E_ + 1] - w[W + 1]) - mD * uD * (w[E_ - 1] - w[W - 1])) +
                zy4 * (mU * vU * (w[N_ + 1] - w[S + 1]) - mD * vD * (w[N_ - 1] - w[S - 1]));
        T hf = xx12 * ((kp[E_] + kP) * (Tt[E_] - TP) - (kp[W] + kP) * (TP - Tt[W])) +
               yy12 * ((kp[N_] + kP) * (Tt[N_] - TP) - (kp[S] + kP) * (TP - Tt[S])) +
               zz12 * ((kp[U_] + kP) * (Tt[U_] - TP) - (kp[D] + kP) * (TP - Tt[D]));
        out[4][n] = inv + vfX + vfY + vfZ + hf;
      }
    }
  }

  // Solver::updatePrimitiveVariables, Solver.cpp:446-479 (seven passes, in this order).
  void updatePrimitives() {
    double gm1 = P.Gamma - 1, Sc = P.sutherlands_C2 / P.T_0, Sc1 = 1 + Sc, pf = 1 / (gm1 * P.Pr);
    auto &rho = cons[0], &ru = cons[1], &rv = cons[2], &rw = cons[3], &rE = cons[4];
    auto &u = prim[0], &v = prim[1], &w = prim[2], &p = prim[3], &Tt = prim[4];
    using std::pow;
    for (size_t i : interior) u[i] = ru[i] / (rho[i] + 1);
    for (size_t i : interior) v[i] = rv[i] / (rho[i] + 1);
    for (size_t i : interior) w[i] = rw[i] / (rho[i] + 1);
    for (size_t i : interior) p[i] = gm1 * (rE[i] - (rho[i] + 1) / 2 * (u[i] * u[i] + v[i] * v[i] + w[i] * w[i]));
    for (size_t i : interior) Tt[i] = (P.Gamma * p[i] - rho[i]) / (1 + rho[i]);
    for (size_t i : interior) mu[i] = pow(1 + Tt[i], 1.5) * Sc1 / (P.Re * (Tt[i] + Sc1));
    for (size_t i : interior) kappa[i] = mu[i] * pf;
  }

  // ---------------- boundary conditions ----------------
  void adjacent(const Edge& e, size_t idx, size_t& a1, size_t& a2) const {  // Boundary.cpp:74-108
    size_t s = e.axis == 0 ? NJ * NK : e.axis == 1 ? NK : 1;
    if (e.side == 0) {
      a1 = idx + s;
      a2 = idx + s * 2;
    } else {
      a1 = idx - s;
      a2 = idx - s * 2;
    }
  }
  size_t periodicIndex(const Edge& e, size_t idx) const {  // Boundary.cpp:111-133
    size_t i, j, kk;
    ijk(idx, i, j, kk);
    if (e.axis == 0) i = e.side == 0 ? NI - 2 : 1;
    if (e.axis == 1) j = e.side == 0 ? NJ - 2 : 1;
    if (e.axis == 2) kk = e.side == 0 ? NK - 2 : 1;
    return id(i, j, kk);
  }
  template <class F>
  void forOwned(const Edge& e, F f) {
    for (size_t i = e.owned.iMin; i <= e.owned.iMax; ++i)
      for (size_t j = e.owned.jMin; j <= e.owned.jMax; ++j)
        for (size_t kk = e.owned.kMin; kk <= e.owned.kMax; ++kk) f(i, j, kk, id(i, j, kk));
  }

  void applyEdge(const Edge& e, double t) {
    auto& rho = cons[0];
    if (e.bc == BC_INLET) {  // InletBoundary::applyBoundaryCondition, Boundary.cpp:250-296
      forOwned(e, [&](size_t, size_t, size_t, size_t idx) {
        size_t a1, a2;
        adjacent(e, idx, a1, a2);
        rho[idx] = 2 * rho[a1] - rho[a2];
      });
      inletFilter(e);
      const double ramp = std::min(1., t / 10.) * P.M_0;
      const bool profiled = e.axis == 0 && !inflowProfile.empty();
      forOwned(e, [&](size_t, size_t j, size_t kk, size_t idx) {
        T vel = T(ramp);
        if (profiled) vel = vel * inflowProfile[j * NK + kk];
        if (e.side == 1) vel = vel * -1.0;
        T uu = T(0.0), vv = T(0.0), ww = T(0.0);
        if (e.axis == 0) uu = vel;
        if (e.axis == 1) vv = vel;
        if (e.axis == 2) ww = vel;
        T r = rho[idx];
        T Tt = T(0.0);
        T p = (Tt * (1 + r) + r) / P.Gamma;
        T pr[5] = {uu, vv, ww, p, Tt}, cv[5], m, kap;
        deriveConserved(pr, cv);
        deriveTransport(pr, m, kap);
        setAll(idx, cv, pr, m, kap);
      });
    } else if (e.bc == BC_OUTLET) {  // OutletBoundary::applyBoundaryCondition, Boundary.cpp:304-336
      forOwned(e, [&](size_t, size_t, size_t, size_t idx) {
        size_t a1, a2;
        adjacent(e, idx, a1, a2);
        T r = 2 * cons[0][a1] - cons[0][a2];
        T ru = 2 * cons[1][a1] - cons[1][a2];
        T rv = 2 * cons[2][a1] - cons[2][a2];
        T rw = 2 * cons[3][a1] - cons[3][a2];
        T p = T(0.0);
        T u = ru / (1 + r), v = rv / (1 + r), w = rw / (1 + r);
        T Tt = (P.Gamma * p - r) / (1 + r);
        T rE = p / (P.Gamma - 1) + (1 + r) / 2 * (u * u + v * v + w * w);
        T pr[5] = {u, v, w, p, Tt}, cv[5] = {r, ru, rv, rw, rE}, m, kap;
        deriveTransport(pr, m, kap);
        setAll(idx, cv, pr, m, kap);
      });
    } else if (e.bc == BC_PERIODIC) {  // PeriodicBoundary::applyBoundaryCondition, Boundary.cpp:344-367
      forOwned(e, [&](size_t, size_t, size_t, size_t idx) {
        size_t o = periodicIndex(e, idx);
        for (int f = 0; f < 5; ++f) cons[f][idx] = cons[f][o];
        for (int f = 0; f < 5; ++f) prim[f][idx] = prim[f][o];
        mu[idx] = mu[o];
        kappa[idx] = kappa[o];
      });
    } else {  // SymmetryBoundary::applyBoundaryCondition, Boundary.cpp:377-417
      forOwned(e, [&](size_t, size_t, size_t, size_t idx) {
        size_t a1, a2;
        adjacent(e, idx, a1, a2);
        T u = prim[0][a2], v = prim[1][a2], w = prim[2][a2];
        if (e.axis == 0) u = -prim[0][a2];
        if (e.axis == 1) v = -prim[1][a2];
        if (e.axis == 2) w = -prim[2][a2];
        T pr[5] = {u, v, w, prim[3][a2], prim[4][a2]}, cv[5], m, kap;
        deriveConserved(pr, cv);
        deriveTransport(pr, m, kap);
        setAll(idx, cv, pr, m, kap);
      });
    }
  }

  void inletFilter(const Edge& e) {  // InletBoundary::filterInletDensity, Boundary.cpp:142-245
    auto& rho = cons[0];
    std::vector<T> vals;
    std::vector<size_t> nodes;
    const Box& o = e.owned;
    auto one = [&](size_t c, size_t pA, size_t mA, bool hasPA, bool hasMA, size_t pB, size_t mB, bool hasPB,
                   bool hasMB) {
      T f = T(0.0);
      unsigned nn = 0;
      if (hasPA) {
        f += rho[pA];
        ++nn;
      }
      if (hasMA) {
        f += rho[mA];
        ++nn;
      }
      if (hasPB) {
        f += rho[pB];
        ++nn;
      }
      if (hasMB) {
        f += rho[mB];
        ++nn;
      }
      f += nn * rho[c];
      f /= 2 * nn;
      vals.push_back(f);
      nodes.push_back(c);
    };
    if (e.axis == 0) {
      size_t i = o.iMin;
      for (size_t j = o.jMin; j <= o.jMax; ++j)
        for (size_t kk = o.kMin; kk <= o.kMax; ++kk)
          one(id(i, j, kk), id(i, j + 1, kk), id(i, j - 1, kk), j < o.jMax, j > o.jMin, id(i, j, kk + 1),
              id(i, j, kk - 1), kk < o.kMax, kk > o.kMin);
    } else if (e.axis == 1) {
      size_t j = o.jMin;
      for (size_t i = o.iMin; i <= o.iMax; ++i)
        for (size_t kk = o.kMin; kk <= o.kMax; ++kk)
          one(id(i, j, kk), id(i + 1, j, kk), id(i - 1, j, kk), i < o.iMax, i > o.iMin, id(i, j, kk + 1),
              id(i, j, kk - 1), kk < o.kMax, kk > o.kMin);
    } else {
      size_t kk = o.kMin;
      for (size_t i = o.iMin; i <= o.iMax; ++i)
        for (size_t j = o.jMin; j <= o.jMax; ++j)
          one(id(i, j, kk), id(i + 1, j, kk), id(i - 1, j, kk), i < o.iMax, i > o.iMin, id(i, j + 1, kk),
              id(i, j - 1, kk), j < o.jMax, j > o.jMin);
    }
    for (size_t q = 0; q < nodes.size(); ++q) rho[nodes[q]] = vals[q];
  }

  // ImmersedBoundary::applyBoundaryCondition, Boundary.cpp:427-457.
  void applyBody(Body& b) {
    // filterClosestFluidNodes, Boundary.cpp:618-652
    {
      std::vector<T> fr, fe;
      const size_t sI = NJ * NK, sJ = NK;
      for (size_t n : b.filter) {
        const auto& r = cons[0];
        const auto& e = cons[4];
        fr.push_back((6 * r[n] + r[n + sI] + r[n - sI] + r[n + sJ] + r[n - sJ] + r[n + 1] + r[n - 1]) / 12);
        fe.push_back((6 * e[n] + e[n + sI] + e[n - sI] + e[n + sJ] + e[n - sJ] + e[n + 1] + e[n - 1]) / 12);
      }
      for (size_t q = 0; q < b.filter.size(); ++q) {
        cons[0][b.filter[q]] = fr[q];
        cons[4][b.filter[q]] = fe[q];
      }
    }
    for (const Ghost& g : b.ghosts) {
      Box sb = surrounding(g.ip);
      size_t cs[8];
      corners(sb, cs);
      T val[5][8];
      double px[8], py[8], pz[8];
      bool gf[8];
      bool allFluid = true;
      std::vector<V3> normals;
      for (int c = 0; c < 8; ++c) {  // setInterpolationValues, Boundary.cpp:697-728
        uint8_t t = type[cs[c]];
        gf[c] = false;
        if (t == FluidInterior || t == FluidEdge || t == FluidGhost) {
          for (int f = 0; f < 5; ++f) val[f][c] = cons[f][cs[c]];
          size_t i, j, kk;
          ijk(cs[c], i, j, kk);
          V3 p = pos(i, j, kk);
          px[c] = p.x;
          py[c] = p.y;
          pz[c] = p.z;
        } else if (t == SolidGhost) {
          gf[c] = true;
          allFluid = false;
          const Ghost& og = b.ghosts.at(b.ghostMap.at(cs[c]));
          V3 nrm = og.ip - og.bi;
          nrm = nrm / nrm.length();
          normals.push_back(nrm);
          for (int f = 0; f < 5; ++f) val[f][c] = T(0.0);
          px[c] = og.bi.x;
          py[c] = og.bi.y;
          pz[c] = og.bi.z;
        } else {
          throw std::logic_error("Impossible situation. Found solid node around image point.");
        }
      }
      T ipv[5];
      if (allFluid) {  // simplifiedInterpolation, Boundary.cpp:732-757
        V3 lo = pos(sb.iMin, sb.jMin, sb.kMin);
        V3 rel = g.ip - lo;
        for (int f = 0; f < 5; ++f) {
          const T* q = val[f];
          T a01 = q[0] + (q[1] - q[0]) * rel.z / dz;
          T a23 = q[2] + (q[3] - q[2]) * rel.z / dz;
          T a45 = q[4] + (q[5] - q[4]) * rel.z / dz;
          T a67 = q[6] + (q[7] - q[6]) * rel.z / dz;
          T a0123 = a01 + (a23 - a01) * rel.y / dy;
          T a4567 = a45 + (a67 - a45) * rel.y / dy;
          ipv[f] = a0123 + (a4567 - a0123) * rel.x / dx;
        }
      } else {  // Vandermonde systems, Boundary.cpp:788-849
        double VD[8][8], VN[8][8];
        for (int r = 0; r < 8; ++r) {
          double row[8] = {1, px[r], py[r], pz[r], px[r] * py[r], px[r] * pz[r], py[r] * pz[r], px[r] * py[r] * pz[r]};
          for (int c = 0; c < 8; ++c) VD[r][c] = VN[r][c] = row[c];
        }
        size_t cnt = 0;
        for (int r = 0; r < 8; ++r)
          if (gf[r]) {
            const V3& nv = normals[cnt];
            VN[r][0] = 0;
            VN[r][1] = nv.x;
            VN[r][2] = nv.y;
            VN[r][3] = nv.z;
            VN[r][4] = px[r] * nv.y + py[r] * nv.x;
            VN[r][5] = px[r] * nv.z + pz[r] * nv.x;
            VN[r][6] = py[r] * nv.z + pz[r] * nv.y;
            VN[r][7] = px[r] * py[r] * nv.z + px[r] * pz[r] * nv.y + py[r] * pz[r] * nv.x;
            ++cnt;
          }
        const double X = g.ip.x, Y = g.ip.y, Z = g.ip.z;
        if constexpr (std::is_same<T, double>::value) {
          if (exactImageSolve) {
            for (int f = 0; f < 5; ++f) ipv[f] = solveExtended(f == 0 || f == 4, px, py, pz, gf, normals, val[f], X, Y, Z);
            goto ghost_value;
          }
        }
        {
        oracle_lu::FullPivLU<8> luD, luN;
        luD.compute(VD);
        luN.compute(VN);
        for (int f = 0; f < 5; ++f) {
          T rhs[8], co[8];
          for (int c = 0; c < 8; ++c) rhs[c] = val[f][c];
          if (f == 0 || f == 4)
            luN.solve(rhs, co);
          else
            luD.solve(rhs, co);
          ipv[f] = co[0] + co[1] * X + co[2] * Y + co[3] * Z + co[4] * X * Y + co[5] * X * Z + co[6] * Y * Z +
                   co[7] * X * Y * Z;
        }
        }
      }
    ghost_value:
      // getGhostNodeBCVariables, Boundary.cpp:777-785
      T gc[5] = {ipv[0], -ipv[1], -ipv[2], -ipv[3], ipv[4]}, gp[5], m, kap;
      derivePrimitive(gc, gp);
      deriveTransport(gp, m, kap);
      setAll(id(g.i, g.j, g.k), gc, gp, m, kap);
    }
  }

  // Extended-precision counterpart of populateVandermonde* + trilinearInterpolation (Boundary.cpp:788-834):
  // the matrix entries (products of the reference's double positions and normals), the solve (Gaussian
  // elimination with partial pivoting) and the polynomial are all evaluated in long double and rounded
  // once to double. Rounding the raw-coordinate entries to double already perturbs the interpolant by
  // about cond(V) * 1e-16, so the entries must be formed in extended precision as well.
  static double solveExtended(bool neumann, const double (&px)[8], const double (&py)[8], const double (&pz)[8],
                              const bool (&gf)[8], const std::vector<V3>& normals, const double (&v)[8], double X,
                              double Y, double Z) {
    long double A[8][9];
    size_t cnt = 0;
    for (int r = 0; r < 8; ++r) {
      const long double x = px[r], y = py[r], z = pz[r];
      if (neumann && gf[r]) {
        const long double nx = normals[cnt].x, ny = normals[cnt].y, nz = normals[cnt].z;
        ++cnt;
        const long double row[8] = {0, nx, ny, nz, x * ny + y * nx, x * nz + z * nx, y * nz + z * ny,
                                    x * y * nz + x * z * ny + y * z * nx};
        for (int c = 0; c < 8; ++c) A[r][c] = row[c];
      } else {
        const long double row[8] = {1, x, y, z, x * y, x * z, y * z, x * y * z};
        for (int c = 0; c < 8; ++c) A[r][c] = row[c];
      }
      A[r][8] = v[r];
    }
    for (int c = 0; c < 8; ++c) {
      int p = c;
      for (int r = c + 1; r < 8; ++r)
        if (std::fabs(A[r][c]) > std::fabs(A[p][c])) p = r;
      for (int q = 0; q < 9; ++q) std::swap(A[c][q], A[p][q]);
      for (int r = c + 1; r < 8; ++r) {
        const long double m = A[r][c] / A[c][c];
        for (int q = c; q < 9; ++q) A[r][q] -= m * A[c][q];
      }
    }
    long double co[8];
    for (int r = 7; r >= 0; --r) {
      long double s = A[r][8];
      for (int q = r + 1; q < 8; ++q) s -= A[r][q] * co[q];
      co[r] = s / A[r][r];
    }
    const long double x = X, y = Y, z = Z;
    return double(co[0] + co[1] * x + co[2] * y + co[3] * z + co[4] * x * y + co[5] * x * z + co[6] * y * z +
                  co[7] * x * y * z);
  }

  // Mesh::applyAllBoundaryConditions, Mesh.cpp:155-167.
  void applyAllBoundaryConditions(double t) {
    for (const Edge& e : edges) applyEdge(e, t);
    for (Body& b : bodies) applyBody(b);
  }

  // Mesh::checkFilterCondition / applyFilter_ifAppropriate, Mesh.cpp:85-140.
  bool filterNow(unsigned long timeLevel, double t) const {
    size_t counter = 0;
    for (double ct : P.filterIntervalChangeTimes)
      if (t > ct) ++counter;
    if (counter < P.filterIntervals.size()) {
      unsigned iv = P.filterIntervals.at(counter);
      if (iv > 0 && (timeLevel + 1) % iv == 0) return true;
    }
    return false;
  }
  void applyFilterIfAppropriate(unsigned long timeLevel, double t) {
    if (!filterNow(timeLevel, t)) return;
    std::vector<T>& f = cons[0];
    std::vector<T>& tmp = old[0];
    for (const Edge& e : edges) forOwned(e, [&](size_t, size_t, size_t, size_t idx) { tmp[idx] = f[idx]; });
    for (size_t idx : solidGhost) tmp[idx] = f[idx];
    const size_t sI = NJ * NK, sJ = NK;
    for (size_t n : interior) tmp[n] = (6 * f[n] + f[n + sI] + f[n - sI] + f[n + sJ] + f[n - sJ] + f[n + 1] + f[n - 1]) / 12;
    f.swap(tmp);
  }

  T normOfChange(const std::vector<T>& o, const std::vector<T>& n) const {  // Mesh.cpp:171-178
    T s = T(0.0);
    using std::pow;
    using std::sqrt;
    for (size_t i : interior) s += pow(o[i] - n[i], 2);
    return sqrt(dx * dy * dz * s);
  }

  // Solver::marchTimeStep, Solver.cpp:130-167.
  void marchTimeStep(double& t, unsigned long& timeLevel) {
    using std::isfinite;
    for (int f = 0; f < 5; ++f)
      for (size_t i = 0; i < N; ++i)
        if (!isfinite(val(cons[f][i]))) nonFinite = true;
    applyFilterIfAppropriate(timeLevel, t);
    for (int f = 0; f < 5; ++f) cons[f].swap(old[f]);
    const double d = val(dt);
    const T dT = dt;
    rhs(old, k[0]);
    intermediate(k[0], dT / 2);
    updatePrimitives();
    applyAllBoundaryConditions(t + d / 2);
    rhs(cons, k[1]);
    intermediate(k[1], dT / 2);
    updatePrimitives();
    applyAllBoundaryConditions(t + d / 2);
    rhs(cons, k[2]);
    intermediate(k[2], dT);
    updatePrimitives();
    applyAllBoundaryConditions(t + d);
    rhs(cons, k[3]);
    finalStep();
    updatePrimitives();
    applyAllBoundaryConditions(t + d);
    storeNorms();
    t += d;
    ++timeLevel;
    ++stepCounter;
    updateTimeStepSize(t);
  }
  void intermediate(std::vector<T>* kk, const T& inc) {  // Solver.cpp:422-442
    for (int f = 0; f < 5; ++f)
      for (size_t i : interior) cons[f][i] = old[f][i] + inc * kk[f][i];
  }
  void finalStep() {  // Solver.cpp:483-507
    T fac = dt / 6;
    for (int f = 0; f < 5; ++f)
      for (size_t i : interior) {
        T res = fac * (k[0][f][i] + 2 * k[1][f][i] + 2 * k[2][f][i] + k[3][f][i]);
        cons[f][i] = old[f][i] + res;
      }
  }
  void storeNorms() {  // Solver.cpp:510-530
    if (P.convHistory != 0) normHistory(0);
    if (P.convHistory == 2)
      for (int f = 1; f < 5; ++f) normHistory(f);
  }
  void normHistory(int f) { normHist[f].push_back(val(normOfChange(old[f], cons[f]))); }

  // The adjoint's objective term: the x-force of the pressure on the bodies, -dA sum_g p(U_g) n_x(g) over
  // the ghost nodes (p from the ghost's conserved values, as the primitive variables are derived; n: the
  // body's unit normal at the ghost's body-intercept point, in the body's cross-section for cylinders;
  // dA = (dx dy dz)^(2/3)).
  T forceX() const {
    const double dA = std::pow(dx * dy * dz, 2.0 / 3.0);
    T s = T(0.0);
    for (const Body& b : bodies)
      for (const Ghost& g : b.ghosts) {
        double d[3] = {g.bi.x - (b.sphere ? b.s.cx : b.c.cx), g.bi.y - (b.sphere ? b.s.cy : b.c.cy),
                       g.bi.z - (b.sphere ? b.s.cz : b.c.cz)};
        if (!b.sphere) d[b.c.axis] = 0;
        const double len = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
        const double nx = len > 0 ? d[0] / len : 0.0;
        const size_t n = id(g.i, g.j, g.k);
        const T rho = cons[0][n], r1 = 1.0 / (rho + 1.0);
        const T u = cons[1][n] * r1, v = cons[2][n] * r1, w = cons[3][n] * r1;
        const T p = (P.Gamma - 1) * (cons[4][n] - (rho + 1.0) * 0.5 * (u * u + v * v + w * w));
        s += -dA * nx * p;
      }
    return s;
  }

  // Level-0 state of a run from a given conserved field (every node): the primitive and transport values
  // are derived from it at every node; the other buffers stay zero.
  void setInitialConserved(const std::vector<T> u0[5]) {
    for (size_t idx = 0; idx < N; ++idx) {
      T cv[5], pr[5], m, kap;
      for (int f = 0; f < 5; ++f) cv[f] = u0[f][idx];
      derivePrimitive(cv, pr);
      deriveTransport(pr, m, kap);
      setAll(idx, cv, pr, m, kap);
    }
  }

  static double val(double x) { return x; }
  template <class U>
  static double val(const U& x) {
    return x.v;
  }
};

}  // namespace nsfo
#endif
