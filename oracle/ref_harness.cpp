// Oracle test infrastructure only (never linked into the product).
//
// Drives the UNMODIFIED reference solver (Frederik-Kris/3D-NS-FSI src/*.cpp, compiled from where they lie
// by oracle/Makefile.ref) on a case file, and dumps what the parity tests compare against:
// node classification, ghost / filter lists, dt and norm histories, and the twelve flow fields.
//
// The reference hard-codes its case in Mesh::setupBoundaries (Mesh.cpp:25-58) and its initial condition
// in Solver::applyStagnation_IC (Solver.cpp:31-51). To run other cases without editing the reference, this
// harness fills the private boundary collections itself (same claim order as Mesh.cpp:33-38, same spacing
// rules as Mesh.cpp:44-49), then calls the reference's own Mesh::categorizeNodes, sets the initial
// condition through the reference's own derive* functions (FlowVariableGroupStructs.h:152-186), and calls
// the private Solver::updateTimeStepSize(0). Private members are reached with the standard
// explicit-instantiation access idiom (C++17 [temp.spec]/6), so no reference source is modified.
// case.kind = "shipped" instead calls Solver::initialize() unchanged (the reference's default case).
//
// Usage: ref_runner <case.cfg> <outdir> [--dump s1,s2,...] [--final] [--vtk] [--time W K]
// --vtk: after the run, the reference's OutputManager writes the VTK snapshot, times.dat and the norm
// files of the final state into <outdir>/output.
// The dump loop stops where Simulation::checkStoppingCriterion (Simulation.cpp:34-52) would stop an
// end_time run; --final then also writes that last state as fields_final.bin.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <chrono>
#include <filesystem>
#include <string>
#include <vector>
#include <set>

#include "OutputManager.h"
#include "Solver.h"

// ---- access to private members (explicit-instantiation idiom) -------------------------------------
template <typename Tag, typename Tag::type M>
struct Grab {
  friend typename Tag::type get(Tag) { return M; }
};
struct MeshEdges {
  typedef EdgeBoundaryCollection Mesh::*type;
  friend type get(MeshEdges);
};
template struct Grab<MeshEdges, &Mesh::edgeBoundaries>;
struct MeshBodies {
  typedef ImmersedBoundaryCollection Mesh::*type;
  friend type get(MeshBodies);
};
template struct Grab<MeshBodies, &Mesh::immersedBoundaries>;
struct SolverUpdateDt {
  typedef void (Solver::*type)(double);
  friend type get(SolverUpdateDt);
};
template struct Grab<SolverUpdateDt, &Solver::updateTimeStepSize>;
struct BodyGhosts {
  typedef vector<GhostNode> ImmersedBoundary::*type;
  friend type get(BodyGhosts);
};
template struct Grab<BodyGhosts, &ImmersedBoundary::ghostNodes>;
struct BodyFilter {
  typedef vector<size_t> ImmersedBoundary::*type;
  friend type get(BodyFilter);
};
template struct Grab<BodyFilter, &ImmersedBoundary::filterNodes>;
struct OutStore {
  typedef void (OutputManager::*type)(const Mesh&, double);
  friend type get(OutStore);
};
template struct Grab<OutStore, &OutputManager::storeCurrentSolution>;
struct OutTimes {
  typedef void (OutputManager::*type)();
  friend type get(OutTimes);
};
template struct Grab<OutTimes, &OutputManager::writeOutputTimes>;
struct OutNorms {
  typedef void (OutputManager::*type)(const ConservedVariablesVectorGroup&);
  friend type get(OutNorms);
};
template struct Grab<OutNorms, &OutputManager::writeConvergenceHistoryFiles>;

// ---- seeded noise shared with the product (splitmix64, Steele/Lea/Flood 2014) ----------------------
static uint64_t splitmix64(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ULL);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}
static double noise_pm1(uint64_t& s) {  // uniform in [-1, 1)
  return 2.0 * (static_cast<double>(splitmix64(s) >> 11) * 0x1.0p-53) - 1.0;
}

static void die(const std::string& m) {
  std::fprintf(stderr, "ref_runner: %s\n", m.c_str());
  std::exit(2);
}

struct FileOut {
  FILE* f;
  explicit FileOut(const std::string& p) : f(std::fopen(p.c_str(), "wb")) {
    if (!f) die("cannot write " + p);
  }
  ~FileOut() { std::fclose(f); }
  void u64(uint64_t v) { std::fwrite(&v, 8, 1, f); }
  void f64(double v) { std::fwrite(&v, 8, 1, f); }
  void raw(const void* p, size_t n) { std::fwrite(p, 1, n, f); }
};

static AxisOrientationEnum axisOf(int a) {
  return a == 0 ? AxisOrientationEnum::x : a == 1 ? AxisOrientationEnum::y : AxisOrientationEnum::z;
}

int main(int argc, char** argv) {
  if (argc < 3) die("usage: ref_runner <case.cfg> <outdir> [--dump s1,s2,...] [--time W K]");
  std::string cfgPath = argv[1], outDir = argv[2];
  std::set<unsigned long> dumps;
  long timeWarm = -1, timeSteps = -1;
  bool dumpFinal = false, writeVtk = false;
  for (int a = 3; a < argc; ++a) {
    if (!std::strcmp(argv[a], "--dump") && a + 1 < argc) {
      std::string s = argv[++a];
      size_t b = 0;
      while (b < s.size()) {
        size_t e = s.find(',', b);
        dumps.insert(std::stoul(s.substr(b, e - b)));
        if (e == std::string::npos) break;
        b = e + 1;
      }
    } else if (!std::strcmp(argv[a], "--final")) {
      dumpFinal = true;
    } else if (!std::strcmp(argv[a], "--vtk")) {
      writeVtk = true;
    } else if (!std::strcmp(argv[a], "--time") && a + 2 < argc) {
      timeWarm = std::stol(argv[++a]);
      timeSteps = std::stol(argv[++a]);
    }
  }

  const ConfigSettings params(cfgPath);
  if (params.errorOccurred) die("reference ConfigSettings reported an error");
  Config cfg;
  cfg.readFile(cfgPath.c_str());
  const Setting& cs = cfg.lookup("case");
  std::string kind = cs["kind"].c_str();

  Solver solver(params);
  Mesh& mesh = solver.mesh;
  if (kind == "shipped") {
    solver.initialize();
  } else {
    // Edge boundaries: one type per face, claimed in the reference's order z-min, z-max, y-min, y-max,
    // x-min, x-max (Mesh.cpp:33-38).
    const char* faceKey[3][2] = {{"bc_x_min", "bc_x_max"}, {"bc_y_min", "bc_y_max"}, {"bc_z_min", "bc_z_max"}};
    std::string type[3][2];
    for (int a = 0; a < 3; ++a)
      for (int m = 0; m < 2; ++m) type[a][m] = cs[faceKey[a][m]].c_str();
    auto& edges = mesh.*get(MeshEdges());
    for (int a = 2; a >= 0; --a)
      for (int m = 0; m < 2; ++m) {
        EdgeIndexEnum e = m == 0 ? EdgeIndexEnum::min : EdgeIndexEnum::max;
        const std::string& t = type[a][m];
        if (t == "periodic")
          edges.push_back(std::make_unique<PeriodicBoundary>(axisOf(a), e));
        else if (t == "symmetry")
          edges.push_back(std::make_unique<SymmetryBoundary>(axisOf(a), e));
        else if (t == "inlet")
          edges.push_back(std::make_unique<InletBoundary>(axisOf(a), e, params.M_0));
        else if (t == "outlet")
          edges.push_back(std::make_unique<OutletBoundary>(axisOf(a), e));
        else
          die("unknown boundary type " + t);
      }
    // Spacing and origin offset per boundary type (Mesh.cpp:44-49 comment and code).
    size_t n[3] = {params.NI, params.NJ, params.NK};
    double L[3] = {params.L_x, params.L_y, params.L_z};
    double d[3], off[3];
    for (int a = 0; a < 3; ++a) {
      const std::string& t = type[a][0];
      if (t == "periodic") {
        d[a] = L[a] / (n[a] - 2);
        off[a] = 1;
      } else if (t == "symmetry") {
        d[a] = L[a] / (n[a] - 3);
        off[a] = 1;
      } else {
        d[a] = L[a] / (n[a] - 1);
        off[a] = 0;
      }
    }
    mesh.dx = d[0];
    mesh.dy = d[1];
    mesh.dz = d[2];
    mesh.positionOffset.x = off[0];
    mesh.positionOffset.y = off[1];
    mesh.positionOffset.z = off[2];
    auto& bodies = mesh.*get(MeshBodies());
    if (cs.exists("spheres")) {
      const Setting& sp = cs["spheres"];
      for (int b = 0; b < sp.getLength(); ++b)
        bodies.push_back(std::make_unique<SphereBody>(
            Vector3_d(double(sp[b][0]), double(sp[b][1]), double(sp[b][2])), double(sp[b][3])));
    }
    if (cs.exists("cylinders")) {
      const Setting& cy = cs["cylinders"];
      for (int b = 0; b < cy.getLength(); ++b) {
        std::string ax = cy[b][0].c_str();
        bodies.push_back(std::make_unique<CylinderBody>(
            Vector3_d(double(cy[b][1]), double(cy[b][2]), double(cy[b][3])),
            axisOf(ax == "x" ? 0 : ax == "y" ? 1 : 2), double(cy[b][4])));
      }
    }
    mesh.categorizeNodes(params);

    // Initial condition through the reference's own derive functions, one node at a time.
    std::string ic = cs["ic"].c_str();
    uint64_t seed = cs.exists("seed") ? static_cast<uint64_t>(static_cast<long long>(cs["seed"])) : 0;
    double amp = cs.exists("noise_amp") ? double(cs["noise_amp"]) : 0.0;
    const Vector3_u nn(mesh.NI, mesh.NJ, mesh.NK);
    const Vector3_d sp(mesh.dx, mesh.dy, mesh.dz);
    for (size_t idx = 0; idx < mesh.nNodesTotal; ++idx) {
      double u = 0, v = 0, w = 0, p = 0, T = 0;
      if (ic == "stagnation") {
      } else if (ic == "freestream_noise") {
        u = params.M_0 + amp * noise_pm1(seed);
        v = amp * noise_pm1(seed);
        w = amp * noise_pm1(seed);
      } else if (ic == "tgv") {
        Vector3_d X = getNodePosition(getIndices3D(idx, nn), sp, mesh.positionOffset);
        double M = params.M_0;
        u = M * std::sin(X.x) * std::cos(X.y) * std::cos(X.z);
        v = -M * std::cos(X.x) * std::sin(X.y) * std::cos(X.z);
        w = 0;
        p = M * M / 16 * (std::cos(2 * X.x) + std::cos(2 * X.y)) * (std::cos(2 * X.z) + 2);
        T = 0;
      } else {
        die("unknown ic " + ic);
      }
      PrimitiveVariablesScalars pv(u, v, w, p, T);
      ConservedVariablesScalars cv = deriveConservedVariables(pv, params);
      TransportPropertiesScalars tv = deriveTransportProperties(pv, params);
      AllFlowVariablesArrayGroup g(mesh.conservedVariables, mesh.primitiveVariables, mesh.transportProperties);
      setFlowVariablesAtNode(idx, cv, pv, tv, g);
    }
    (solver.*get(SolverUpdateDt()))(0);
  }

  // ---- setup dump ----
  {
    FileOut o(outDir + "/setup.bin");
    o.u64(0x4E53465352454631ULL);  // "NSFSREF1"
    o.u64(mesh.NI);
    o.u64(mesh.NJ);
    o.u64(mesh.NK);
    o.f64(mesh.dx);
    o.f64(mesh.dy);
    o.f64(mesh.dz);
    o.f64(mesh.positionOffset.x);
    o.f64(mesh.positionOffset.y);
    o.f64(mesh.positionOffset.z);
    std::vector<uint8_t> types(mesh.nNodesTotal);
    for (size_t i = 0; i < mesh.nNodesTotal; ++i) types[i] = static_cast<uint8_t>(mesh.nodeType(i));
    o.raw(types.data(), types.size());
    auto& bodies = mesh.*get(MeshBodies());
    o.u64(bodies.size());
    for (auto& b : bodies) {
      const vector<GhostNode>& g = (*b).*get(BodyGhosts());
      const vector<size_t>& f = (*b).*get(BodyFilter());
      o.u64(g.size());
      for (const GhostNode& gn : g) {
        o.u64(gn.indices.i);
        o.u64(gn.indices.j);
        o.u64(gn.indices.k);
        o.f64(gn.bodyInterceptPoint.x);
        o.f64(gn.bodyInterceptPoint.y);
        o.f64(gn.bodyInterceptPoint.z);
        o.f64(gn.imagePoint.x);
        o.f64(gn.imagePoint.y);
        o.f64(gn.imagePoint.z);
      }
      o.u64(f.size());
      for (size_t fi : f) o.u64(fi);
    }
    o.f64(solver.dt);
  }

  auto dumpFields = [&](double t, unsigned long level, bool final_ = false) {
    char name[64];
    if (final_)
      std::snprintf(name, sizeof name, "/fields_final.bin");
    else
      std::snprintf(name, sizeof name, "/fields_%06lu.bin", level);
    FileOut o(outDir + name);
    o.f64(t);
    o.u64(level);
    o.f64(solver.dt);
    const Array3D_d* arr[12] = {&mesh.conservedVariables.rho,   &mesh.conservedVariables.rho_u,
                                &mesh.conservedVariables.rho_v, &mesh.conservedVariables.rho_w,
                                &mesh.conservedVariables.rho_E, &mesh.primitiveVariables.u,
                                &mesh.primitiveVariables.v,     &mesh.primitiveVariables.w,
                                &mesh.primitiveVariables.p,     &mesh.primitiveVariables.T,
                                &mesh.transportProperties.mu,   &mesh.transportProperties.kappa};
    for (const Array3D_d* a : arr)
      for (size_t i = 0; i < mesh.nNodesTotal; ++i) o.f64((*a)(i));
  };

  double t = 0;
  ulong timeLevel = 0;
  if (timeSteps >= 0) {
    // Timing mode: warm-up steps, then time exactly K calls of Solver::marchTimeStep.
    for (long s = 0; s < timeWarm; ++s) solver.marchTimeStep(t, timeLevel);
    auto t0 = std::chrono::steady_clock::now();
    for (long s = 0; s < timeSteps; ++s) solver.marchTimeStep(t, timeLevel);
    double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::printf("{\"seconds\": %.9g, \"steps\": %ld, \"nodes\": %zu, \"node_steps_per_s\": %.9g, \"t\": %.17g}\n", sec,
                timeSteps, mesh.nNodesTotal, sec > 0 ? double(mesh.nNodesTotal) * timeSteps / sec : 0.0, t);
    return 0;
  }

  unsigned long lastDump = dumps.empty() ? 0 : *dumps.rbegin();
  FileOut hist(outDir + "/history.bin");
  if (dumps.count(0)) dumpFields(t, 0);
  while (timeLevel < lastDump) {
    if (params.stopCriterion == StopCriterionEnum::end_time && !(t < params.t_end)) break;
    double dtUsed = solver.dt;
    solver.marchTimeStep(t, timeLevel);
    hist.f64(t);
    hist.f64(dtUsed);
    hist.f64(solver.dt);
    const ConservedVariablesVectorGroup& nh = solver.getConvergenceHistory();
    const vector<double>* hv[5] = {&nh.rho, &nh.rho_u, &nh.rho_v, &nh.rho_w, &nh.rho_E};
    for (auto* v : hv) hist.f64(v->empty() ? -1.0 : v->back());
    if (dumps.count(timeLevel)) dumpFields(t, timeLevel);
  }
  if (dumpFinal) dumpFields(t, timeLevel, true);
  if (writeVtk) {
    // The reference's own output writer on the final state: out.vtk.0, times.dat and norm_*.dat in
    // <outdir>/output (OutputManager writes to ./output).
    std::filesystem::create_directories(outDir + "/output");
    std::filesystem::current_path(outDir);
    OutputManager out(params);
    (out.*get(OutStore()))(mesh, t);
    (out.*get(OutTimes()))();
    (out.*get(OutNorms()))(solver.getConvergenceHistory());
  }
  return 0;
}
