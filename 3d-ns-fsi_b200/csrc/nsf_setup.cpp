// Host-side mesh setup: boundary claims, node classification, immersed-body ghost / filter lists,
// image points and the initial condition. Runs once per solver, before the first step.
//
// Node classification, ghost lists and image-point cells must be bit-exact with the reference, so every
// floating-point expression here is evaluated in the reference's order and the file is compiled with
// -ffp-contract=off (no fused multiply-add contraction). Reference functions:
//   Mesh::setupBoundaries            src/Mesh.cpp:25-58     (spacing / offset rules, claim order)
//   Mesh::categorizeNodes            src/Mesh.cpp:61-82
//   MeshEdgeBoundary::identifyOwnedNodes  src/Boundary.cpp:18-71
//   {Cylinder,Sphere}Body::identifyRelatedNodes  src/Boundary.cpp:894-917, :1023-1044
//   bounding boxes                   src/Boundary.cpp:938-965, :1056-1072
//   solid / filter scans             src/Boundary.cpp:968-1014, :1075-1103
//   findGhostNodesWithFluidNeighbors src/Boundary.cpp:461-562
//   setImagePointPositions / appendGhostNodes  src/Boundary.cpp:582-615
//   getNormalProbe                   src/Boundary.cpp:920-935, :1047-1053
//   derive{Conserved,Transport}      src/FlowVariableGroupStructs.h:152-186
#include <algorithm>
#include <cmath>
#include <set>

#include "nsf_internal.h"

namespace nsf {

namespace {

struct Vec {
  double x, y, z;
};
inline Vec sub(Vec a, Vec b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline Vec add(Vec a, Vec b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline Vec scale(Vec a, double f) { return {a.x * f, a.y * f, a.z * f}; }
// Vector3_d::length, src/SmallVectors.h:20.
inline double norm3(Vec a) { return std::sqrt(std::pow(a.x, 2) + std::pow(a.y, 2) + std::pow(a.z, 2)); }

inline size_t lin(const HostSetup& s, size_t i, size_t j, size_t k) { return i * s.NJ * s.NK + j * s.NK + k; }

inline Vec posOf(const HostSetup& s, size_t i, size_t j, size_t k) {
  double p[3];
  node_position(s, i, j, k, p);
  return {p[0], p[1], p[2]};
}

// Vector from a ghost node to the closest surface point.
Vec probe(const BodyRec& b, Vec g) {
  Vec c2g = sub(g, Vec{b.c[0], b.c[1], b.c[2]});
  if (!b.sphere) {
    if (b.axis == 0) c2g.x = 0;
    if (b.axis == 1) c2g.y = 0;
    if (b.axis == 2) c2g.z = 0;
  }
  double lengthFactor = (b.r - norm3(c2g)) / norm3(c2g);
  return scale(c2g, lengthFactor);
}

// Does the 18-point stencil around a solid node touch an interior fluid node?
bool touchesInterior(const HostSetup& s, size_t i, size_t j, size_t k) {
  static const int nb[18][3] = {{-1, 0, 0}, {-1, -1, 0}, {-1, 1, 0}, {-1, 0, -1}, {-1, 0, 1}, {1, 0, 0},
                                {1, -1, 0}, {1, 1, 0},   {1, 0, -1}, {1, 0, 1},   {0, -1, 0}, {0, -1, -1},
                                {0, -1, 1}, {0, 1, 0},   {0, 1, -1}, {0, 1, 1},   {0, 0, -1}, {0, 0, 1}};
  for (auto& o : nb) {
    long a = long(i) + o[0], b = long(j) + o[1], c = long(k) + o[2];
    if (a < 0 || b < 0 || c < 0 || a >= long(s.NI) || b >= long(s.NJ) || c >= long(s.NK)) continue;
    if (s.type[lin(s, a, b, c)] == FLUID_INTERIOR) return true;
  }
  return false;
}

nsf_status classifyBody(const nsf_config& cfg, HostSetup& s, BodyRec& b, std::string& err) {
  const size_t layer = 2;
  const double dx = s.d[0], dy = s.d[1], dz = s.d[2];
  size_t rad[3] = {static_cast<size_t>(std::ceil(b.r / dx)) + 1 + layer,
                   static_cast<size_t>(std::ceil(b.r / dy)) + 1 + layer,
                   static_cast<size_t>(std::ceil(b.r / dz)) + 1 + layer};
  // The reference rounds c/d without the origin offset and never clamps the box.
  double cidx[3] = {std::round(b.c[0] / dx), std::round(b.c[1] / dy), std::round(b.c[2] / dz)};
  size_t n[3] = {s.NI, s.NJ, s.NK};
  long lo[3], hi[3];
  for (int a = 0; a < 3; ++a) {
    if (!b.sphere && a == b.axis) {
      lo[a] = 0;
      hi[a] = long(n[a]) - 1;
      continue;
    }
    if (cidx[a] < 0) {
      err = "immersed body centre lies outside the mesh";
      return NSF_ERR_GEOMETRY;
    }
    size_t cc = static_cast<size_t>(cidx[a]);
    lo[a] = long(cc) - long(rad[a]);
    hi[a] = long(cc) + long(rad[a]);
    if (lo[a] < 0 || hi[a] > long(n[a]) - 1) {
      err = "immersed body (with its filter layer) is too close to a mesh face: the reference's bounding box "
            "would leave the mesh";
      return NSF_ERR_GEOMETRY;
    }
  }
  std::vector<size_t> solids;
  const double fwSphere = layer * std::max({dx, dy, dz});
  for (size_t i = lo[0]; i <= size_t(hi[0]); ++i)
    for (size_t j = lo[1]; j <= size_t(hi[1]); ++j)
      for (size_t k = lo[2]; k <= size_t(hi[2]); ++k) {
        Vec p = posOf(s, i, j, k);
        double dist, fw;
        if (b.sphere) {
          dist = std::sqrt(std::pow(p.x - b.c[0], 2) + std::pow(p.y - b.c[1], 2) + std::pow(p.z - b.c[2], 2));
          fw = fwSphere;
        } else if (b.axis == 0) {
          dist = std::sqrt(std::pow(p.y - b.c[1], 2) + std::pow(p.z - b.c[2], 2));
          fw = layer * std::max(dy, dz);
        } else if (b.axis == 1) {
          dist = std::sqrt(std::pow(p.x - b.c[0], 2) + std::pow(p.z - b.c[2], 2));
          fw = layer * std::max(dx, dz);
        } else {
          dist = std::sqrt(std::pow(p.x - b.c[0], 2) + std::pow(p.y - b.c[1], 2));
          fw = layer * std::max(dx, dy);
        }
        size_t idx = lin(s, i, j, k);
        if (dist < b.r - cfg.machine_precision_buffer) {
          s.type[idx] = SOLID_INACTIVE;
          solids.push_back(idx);
        } else if (dist < b.r + fw && s.type[idx] == FLUID_INTERIOR) {
          b.filter.push_back(idx);
        }
      }
  for (size_t idx : solids) {
    size_t i = idx / (s.NJ * s.NK), j = idx % (s.NJ * s.NK) / s.NK, k = idx % s.NK;
    if (touchesInterior(s, i, j, k)) {
      b.ghostIndex[idx] = b.ghosts.size();
      b.ghosts.push_back(GhostRec{i, j, k, {0, 0, 0}, {0, 0, 0}});
      s.type[idx] = SOLID_GHOST;
    }
  }
  // Image points, repeated until no solid inactive node surrounds any image point (the well-defined
  // cylinder form of the closure loop; the sphere form at Boundary.cpp:1039-1043 is undefined
  // behaviour whenever the loop body runs, so closureAdded is reported for the caller to check).
  size_t first = 0;
  for (;;) {
    std::vector<GhostRec> fresh;
    for (size_t g = first; g < b.ghosts.size(); ++g) {
      GhostRec& gh = b.ghosts[g];
      Vec gp = posOf(s, gh.i, gh.j, gh.k);
      Vec np = probe(b, gp);
      Vec bi = add(gp, np);
      Vec ip = add(bi, np);
      gh.bi[0] = bi.x;
      gh.bi[1] = bi.y;
      gh.bi[2] = bi.z;
      gh.ip[0] = ip.x;
      gh.ip[1] = ip.y;
      gh.ip[2] = ip.z;
      Box box;
      if (!surrounding_box(s, gh.ip, box)) {
        err = "an image point lies outside the mesh (the reference reads out of range there)";
        return NSF_ERR_GEOMETRY;
      }
      int64_t cs[8];
      box_corners(s, box, cs);
      for (int64_t c : cs)
        if (s.type[c] == SOLID_INACTIVE) {
          size_t a = c / (s.NJ * s.NK), bb = c % (s.NJ * s.NK) / s.NK, cc = c % s.NK;
          fresh.push_back(GhostRec{a, bb, cc, {0, 0, 0}, {0, 0, 0}});
          s.type[c] = SOLID_GHOST;
        }
    }
    if (fresh.empty()) break;
    first = b.ghosts.size();
    for (auto& g : fresh) {
      b.ghostIndex[lin(s, g.i, g.j, g.k)] = b.ghosts.size();
      b.ghosts.push_back(g);
    }
    b.closureAdded += fresh.size();
  }
  return NSF_OK;
}

}  // namespace

bool surrounding_box(const HostSetup& s, const double p[3], Box& b) {
  double raw[3] = {std::ceil(p[0] / s.d[0]) + s.off[0], std::ceil(p[1] / s.d[1]) + s.off[1],
                   std::ceil(p[2] / s.d[2]) + s.off[2]};
  size_t n[3] = {s.NI, s.NJ, s.NK}, nx[3];
  for (int a = 0; a < 3; ++a) {
    if (!(raw[a] >= 0)) return false;
    nx[a] = static_cast<size_t>(raw[a]);
    nx[a] = std::max<size_t>(nx[a], 1);
    nx[a] = std::min<size_t>(nx[a], n[a]);
    if (nx[a] > n[a] - 1) return false;  // the reference clamps to n, one past the last node
  }
  b = Box{nx[0] - 1, nx[0], nx[1] - 1, nx[1], nx[2] - 1, nx[2]};
  return true;
}

void box_corners(const HostSetup& s, const Box& b, int64_t out[8]) {
  size_t is[2] = {b.i0, b.i1}, js[2] = {b.j0, b.j1}, ks[2] = {b.k0, b.k1};
  int q = 0;
  for (size_t i : is)
    for (size_t j : js)
      for (size_t k : ks) out[q++] = int64_t(lin(s, i, j, k));
}

nsf_status build_setup(const nsf_config& cfg, HostSetup& s, std::string& err) {
  nsf_config c = cfg;
  if (c.shipped_case) {  // Mesh::setupBoundaries as shipped: Mesh.cpp:33-55
    c.bc[2][0] = c.bc[2][1] = NSF_BC_PERIODIC;
    c.bc[1][0] = c.bc[1][1] = NSF_BC_SYMMETRY;
    c.bc[0][0] = NSF_BC_INLET;
    c.bc[0][1] = NSF_BC_OUTLET;
    c.n_spheres = 0;
    c.n_cylinders = 1;
    c.cylinders[0] = nsf_cylinder{2, c.lx / 4, c.ly / 2, 0, c.ly / 10};
  }
  s.NI = c.NI;
  s.NJ = c.NJ;
  s.NK = c.NK;
  s.N = s.NI * s.NJ * s.NK;
  size_t n[3] = {s.NI, s.NJ, s.NK};
  double L[3] = {c.lx, c.ly, c.lz};
  for (int a = 0; a < 3; ++a) {
    int lo = c.bc[a][0], hi = c.bc[a][1];
    bool pair = (lo == NSF_BC_PERIODIC) == (hi == NSF_BC_PERIODIC) && (lo == NSF_BC_SYMMETRY) == (hi == NSF_BC_SYMMETRY);
    if (lo < 0 || lo > 3 || hi < 0 || hi > 3 || !pair) {
      err = "boundary types must pair per axis: periodic/periodic, symmetry/symmetry, or inlet/outlet";
      return NSF_ERR_CONFIG;
    }
    size_t minN = lo == NSF_BC_SYMMETRY ? 4 : 3;  // ConfigFile: minimum node counts per BC type
    if (n[a] < minN) {
      err = "too few nodes along an axis for its boundary type";
      return NSF_ERR_CONFIG;
    }
    // Spacing and origin offset: in/out N-1 & 0, periodic N-2 & 1, symmetry N-3 & 1 (Mesh.cpp:44-49).
    if (lo == NSF_BC_PERIODIC) {
      s.d[a] = L[a] / (n[a] - 2);
      s.off[a] = 1;
    } else if (lo == NSF_BC_SYMMETRY) {
      s.d[a] = L[a] / (n[a] - 3);
      s.off[a] = 1;
    } else {
      s.d[a] = L[a] / (n[a] - 1);
      s.off[a] = 0;
    }
  }
  s.type.assign(s.N, FLUID_INTERIOR);
  // Claims: z-min, z-max, y-min, y-max, x-min, x-max; each takes every still-unclaimed node of its plane.
  Box open{0, s.NI - 1, 0, s.NJ - 1, 0, s.NK - 1};
  std::vector<EdgeBC> claims;
  for (int a = 2; a >= 0; --a)
    for (int side = 0; side < 2; ++side) {
      EdgeBC e{a, side, c.bc[a][side], open};
      size_t* lo[3] = {&open.i0, &open.j0, &open.k0};
      size_t* hi[3] = {&open.i1, &open.j1, &open.k1};
      size_t* elo[3] = {&e.owned.i0, &e.owned.j0, &e.owned.k0};
      size_t* ehi[3] = {&e.owned.i1, &e.owned.j1, &e.owned.k1};
      if (side == 0) {
        *ehi[a] = *elo[a];
        ++*lo[a];
      } else {
        *elo[a] = *ehi[a];
        --*hi[a];
      }
      uint8_t t = (e.bc == NSF_BC_INLET || e.bc == NSF_BC_OUTLET) ? FLUID_EDGE : FLUID_GHOST;
      for (size_t i = e.owned.i0; i <= e.owned.i1; ++i)
        for (size_t j = e.owned.j0; j <= e.owned.j1; ++j)
          for (size_t k = e.owned.k0; k <= e.owned.k1; ++k) s.type[lin(s, i, j, k)] = t;
      claims.push_back(e);
    }
  s.edges.assign(claims.rbegin(), claims.rend());

  s.bodies.clear();
  for (int q = 0; q < c.n_spheres; ++q) {
    BodyRec b;
    b.sphere = true;
    b.c[0] = c.spheres[q].cx;
    b.c[1] = c.spheres[q].cy;
    b.c[2] = c.spheres[q].cz;
    b.r = c.spheres[q].r;
    b.axis = -1;
    s.bodies.push_back(b);
  }
  for (int q = 0; q < c.n_cylinders; ++q) {
    BodyRec b;
    b.sphere = false;
    b.c[0] = c.cylinders[q].cx;
    b.c[1] = c.cylinders[q].cy;
    b.c[2] = c.cylinders[q].cz;
    b.r = c.cylinders[q].r;
    b.axis = c.cylinders[q].axis;
    if (b.axis < 0 || b.axis > 2) {
      err = "cylinder axis must be 0, 1 or 2";
      return NSF_ERR_CONFIG;
    }
    s.bodies.push_back(b);
  }
  for (auto& b : s.bodies) {
    if (!(b.r > 0)) {
      err = "body radius must be positive";
      return NSF_ERR_CONFIG;
    }
    nsf_status st = classifyBody(c, s, b, err);
    if (st != NSF_OK) return st;
  }

  // Checks. The reference cannot run a solid inactive node inside an image-point cell (it throws,
  // Boundary.cpp:723-724) nor another body's ghost node there (its ghost lookup, Boundary.cpp:681, throws
  // std::out_of_range); both are refused. Bodies that otherwise reach each other's nodes -- a node filtered
  // by two bodies, a ghost shared by two bodies, a filter stencil or an image-point cell touching another
  // body's ghost or filter nodes -- run in the reference's body order (bodiesInteract). Refused as well: a
  // filter node of one body that a later body made solid, whose stale primitive values (the reference never
  // recomputes them at a filter node) the device does not keep for solid nodes.
  std::vector<int> owner(s.N, -1);
  s.bodiesInteract = false;
  for (size_t q = 0; q < s.bodies.size(); ++q) {
    for (auto& g : s.bodies[q].ghosts) {
      const size_t n = lin(s, g.i, g.j, g.k);
      if (owner[n] >= 0 && owner[n] != int(q)) s.bodiesInteract = true;
      owner[n] = int(q);
    }
    for (size_t f : s.bodies[q].filter) {
      if (s.type[f] != FLUID_INTERIOR) {
        err = "immersed bodies are too close: a filter node of one body lies inside another";
        return NSF_ERR_GEOMETRY;
      }
      if (owner[f] >= 0 && owner[f] != int(q)) s.bodiesInteract = true;
      owner[f] = int(q);
    }
  }
  const long sI = long(s.NJ * s.NK), sJ = long(s.NK);
  for (size_t q = 0; q < s.bodies.size(); ++q) {
    for (size_t f : s.bodies[q].filter)
      for (long o : {sI, -sI, sJ, -sJ, 1L, -1L}) {
        long nb = long(f) + o;
        if (owner[nb] >= 0 && owner[nb] != int(q)) s.bodiesInteract = true;
      }
    for (auto& g : s.bodies[q].ghosts) {
      Box box;
      surrounding_box(s, g.ip, box);
      int64_t cs[8];
      box_corners(s, box, cs);
      for (int64_t cn : cs) {
        uint8_t t = s.type[cn];
        if (t == SOLID_INACTIVE) {
          err = "Impossible situation. Found solid node around image point.";
          return NSF_ERR_GEOMETRY;
        }
        if (t == SOLID_GHOST && !s.bodies[q].ghostIndex.count(size_t(cn))) {
          err = "an image-point cell holds another body's ghost node (the reference's ghost lookup fails there)";
          return NSF_ERR_GEOMETRY;
        }
        if (owner[cn] >= 0 && owner[cn] != int(q)) s.bodiesInteract = true;
      }
    }
  }
  return NSF_OK;
}

// Initial condition (Solver::applyStagnation_IC, Solver.cpp:31-51, generalised): primitive values per
// node, conserved and transport values through deriveConservedVariables / deriveTransportProperties.
// Seeded noise: splitmix64 (Steele, Lea, Flood 2014), three draws (u, v, w) per node in index order,
// mapped to [-1, 1).
void initial_condition(const nsf_config& cfg, const HostSetup& s, std::vector<double>& cons5,
                       std::vector<double>& prim7) {
  const size_t N = s.N;
  cons5.assign(5 * N, 0.0);
  prim7.assign(7 * N, 0.0);
  uint64_t state = cfg.seed;
  auto draw = [&state]() {
    uint64_t z = (state += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    z ^= z >> 31;
    return 2.0 * (static_cast<double>(z >> 11) * 0x1.0p-53) - 1.0;
  };
  const int ic = cfg.shipped_case ? NSF_IC_STAGNATION : cfg.ic;
  const double G = cfg.gamma, M = cfg.m0;
  const double ScPlusOne = 1 + cfg.sutherlands_c2 / cfg.t0;
  for (size_t idx = 0; idx < N; ++idx) {
    double u = 0, v = 0, w = 0, p = 0, T = 0;
    if (ic == NSF_IC_FREESTREAM_NOISE) {
      u = M + cfg.noise_amp * draw();
      v = cfg.noise_amp * draw();
      w = cfg.noise_amp * draw();
    } else if (ic == NSF_IC_TGV) {
      size_t i = idx / (N / s.NI), j = idx % (s.NJ * s.NK) / s.NK, k = idx % s.NK;
      double X[3];
      node_position(s, i, j, k, X);
      u = M * std::sin(X[0]) * std::cos(X[1]) * std::cos(X[2]);
      v = -M * std::cos(X[0]) * std::sin(X[1]) * std::cos(X[2]);
      p = M * M / 16 * (std::cos(2 * X[0]) + std::cos(2 * X[1])) * (std::cos(2 * X[2]) + 2);
    }
    double rho = (G * p - T) / (1 + T);
    cons5[0 * N + idx] = rho;
    cons5[1 * N + idx] = (1 + rho) * u;
    cons5[2 * N + idx] = (1 + rho) * v;
    cons5[3 * N + idx] = (1 + rho) * w;
    cons5[4 * N + idx] = p / (G - 1) + (1 + rho) / 2 * (u * u + v * v + w * w);
    double mu = std::pow(1 + T, 1.5) * ScPlusOne / (cfg.re * (T + ScPlusOne));
    prim7[0 * N + idx] = u;
    prim7[1 * N + idx] = v;
    prim7[2 * N + idx] = w;
    prim7[3 * N + idx] = p;
    prim7[4 * N + idx] = T;
    prim7[5 * N + idx] = mu;
    prim7[6 * N + idx] = mu / ((G - 1) * cfg.pr);
  }
}

}  // namespace nsf
