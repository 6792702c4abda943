// C++ host classes of the B200 time-marching path, mirroring the reference's call surface
// (Frederik-Kris/3D-NS-FSI: ConfigSettings, Simulation, Solver, Mesh, OutputManager) on top of the C ABI in
// include/nsfsi.h. A program written against the reference,
//
//     ConfigSettings params("ConfigFile");        // src/main.cpp:12-20
//     if (params.errorOccurred) return -1;
//     Simulation simulation(params);
//     simulation.run();
//
// compiles unchanged against this header (namespace nsfsi) and runs the time marching on a B200. The
// flow fields stay resident on the device. Snapshots download only the fields the settings save, into
// page-locked buffers, while the march goes on; a worker thread writes each file once its fields have
// landed (SnapshotWriter). Mesh keeps host mirrors for callers that read its arrays (Mesh::syncFromDevice).
//
// Header-only; link with 3d-ns-fsi_b200/lib/libnsfsi.so.
#ifndef NSFSI_HOST_HPP
#define NSFSI_HOST_HPP

#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdint>
#include <deque>
#include <exception>
#include <filesystem>
#include <fstream>
#include <functional>
#include <iomanip>
#include <iostream>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "nsfsi.h"

namespace nsfsi {

using ulong = unsigned long;

// Thrown for any non-zero status of the C ABI (the reference has no error codes; it prints and
// continues or throws std::logic_error).
struct Error : std::runtime_error {
  nsf_status status;
  Error(nsf_status s, const std::string& what) : std::runtime_error(what), status(s) {}
};

inline const char* status_name(nsf_status st) {
  static const char* names[] = {"NSF_OK",         "NSF_ERR_CONFIG",  "NSF_ERR_CUDA", "NSF_ERR_NONFINITE",
                                "NSF_ERR_GEOMETRY", "NSF_ERR_TIMEOUT", "NSF_ERR_ARG",  "NSF_ERR_STATE"};
  return unsigned(st) < 8 ? names[st] : "unknown status";
}

inline void check(nsf_status st, nsf_solver* h, const char* call) {
  if (st != NSF_OK)
    throw Error(st, std::string(call) + ": " + status_name(st) + (h ? std::string(": ") + nsf_last_error(h) : ""));
}

enum class StopCriterionEnum { timesteps, end_time };
enum class ConvHistoryEnum { none, density, all };
enum class NodeTypeEnum : uint8_t { FluidInterior, FluidEdge, FluidGhost, SolidInactive, SolidGhost };

// ConfigSettings (src/ConfigSettings.h:33-80): the parsed ConfigFile. The public members keep the
// reference's names; `raw` is the C struct the library consumes (it also carries the case description).
class ConfigSettings {
 public:
  explicit ConfigSettings(const std::string& filename) {  // ConfigSettings.cpp:11-33
    char err[1024] = {0};
    errorOccurred = nsf_config_load(filename.c_str(), &raw, err, sizeof err) != NSF_OK;
    if (errorOccurred) {
      std::cerr << err << std::endl;
      return;
    }
    mirror();
  }
  explicit ConfigSettings(const nsf_config& c) : raw(c) { mirror(); }

  nsf_config raw{};
  bool errorOccurred = false;
  size_t NI = 0, NJ = 0, NK = 0;
  StopCriterionEnum stopCriterion = StopCriterionEnum::timesteps;
  ulong stopTimeLevel = 0;
  double t_end = 0, convStabilityLimit = 0, viscStabilityLimit = 0, statusReportInterval = 0;
  std::vector<unsigned> filterIntervals;
  std::vector<double> filterIntervalChangeTimes;
  bool saveDensity = false, saveMomentum = false, saveEnergy = false, saveVelocity = false, savePressure = false,
       saveTemperature = false, saveViscosity = false, saveThermalCond = false, saveIC = false, saveFinal = false,
       saveIntervals = false;
  double savePeriod = 0, saveIntervalsStartTime = 0, saveIntervalsEndTime = 0;
  ConvHistoryEnum saveConvergenceHistory = ConvHistoryEnum::none;
  double Gamma = 0, Pr = 0, R = 0, Re = 0, sutherlands_C1 = 0, sutherlands_C2 = 0, M_0 = 0, T_0 = 0;
  double L_x = 0, L_y = 0, L_z = 0, machinePrecisionBuffer = 0;

 private:
  void mirror() {
    const nsf_config& c = raw;
    NI = size_t(c.NI);
    NJ = size_t(c.NJ);
    NK = size_t(c.NK);
    stopCriterion = c.stop_criterion == 1 ? StopCriterionEnum::end_time : StopCriterionEnum::timesteps;
    stopTimeLevel = ulong(c.stop_time_level);
    t_end = c.t_end;
    convStabilityLimit = c.conv_stability_limit;
    viscStabilityLimit = c.visc_stability_limit;
    filterIntervals.assign(c.filter_intervals, c.filter_intervals + c.n_filter_intervals);
    filterIntervalChangeTimes.assign(c.filter_change_times, c.filter_change_times + c.n_filter_change_times);
    statusReportInterval = c.status_report_interval;
    saveDensity = c.save_density;
    saveMomentum = c.save_momentum;
    saveEnergy = c.save_energy;
    saveVelocity = c.save_velocity;
    savePressure = c.save_pressure;
    saveTemperature = c.save_temperature;
    saveViscosity = c.save_viscosity;
    saveThermalCond = c.save_thermal_cond;
    saveIC = c.save_ic;
    saveFinal = c.save_final;
    saveIntervals = c.save_intervals;
    savePeriod = c.save_period;
    saveIntervalsStartTime = c.save_intervals_start_time;
    saveIntervalsEndTime = c.save_intervals_end_time;
    saveConvergenceHistory = ConvHistoryEnum(c.conv_history);
    Gamma = c.gamma;
    Pr = c.pr;
    R = c.r_gas;
    Re = c.re;
    sutherlands_C1 = c.sutherlands_c1;
    sutherlands_C2 = c.sutherlands_c2;
    M_0 = c.m0;
    T_0 = c.t0;
    L_x = c.lx;
    L_y = c.ly;
    L_z = c.lz;
    machinePrecisionBuffer = c.machine_precision_buffer;
  }
};

// Host mirror of one field (Array3D_d, src/Array3D.h:20-122): k fastest.
struct Array3D_d {
  size_t NI = 0, NJ = 0, NK = 0;
  std::vector<double> data;
  double operator()(size_t i, size_t j, size_t k) const { return data[i * NJ * NK + j * NK + k]; }
  double at(size_t i, size_t j, size_t k) const { return data.at(i * NJ * NK + j * NK + k); }
  double operator()(size_t n) const { return data[n]; }
};
struct Vector3_d {
  double x = 0, y = 0, z = 0;
};
struct ConservedVariablesArrayGroup {
  Array3D_d rho, rho_u, rho_v, rho_w, rho_E;
};
struct PrimitiveVariablesArrayGroup {
  Array3D_d u, v, w, p, T;
};
struct TransportPropertiesArrayGroup {
  Array3D_d mu, kappa;
};
struct ConservedVariablesVectorGroup {  // norm histories (FlowVariableGroupStructs.h)
  std::vector<double> rho, rho_u, rho_v, rho_w, rho_E;
};

// Mesh (src/Mesh.h:23-93): sizes, spacing, node types and host mirrors of the flow fields.
class Mesh {
 public:
  size_t NI = 0, NJ = 0, NK = 0, nNodesTotal = 0;
  double dx = 0, dy = 0, dz = 0;
  Vector3_d positionOffset;
  // Host mirrors of the device fields, refreshed by syncFromDevice.
  mutable ConservedVariablesArrayGroup conservedVariables;
  mutable PrimitiveVariablesArrayGroup primitiveVariables;
  mutable TransportPropertiesArrayGroup transportProperties;
  std::vector<uint8_t> nodeTypes;

  NodeTypeEnum nodeType(size_t i, size_t j, size_t k) const { return NodeTypeEnum(nodeTypes[i * NJ * NK + j * NK + k]); }

  // Copy the current fields (bit f of `fieldMask` = field f, NSF_RHO..NSF_KAPPA) from the device into
  // the host mirrors, one synchronising download; the mirrors of fields not asked for are left as they are.
  void syncFromDevice(uint32_t fieldMask = (1u << NSF_NUM_FIELDS) - 1) const {
    fieldMask &= (1u << NSF_NUM_FIELDS) - 1;
    size_t nf = 0;
    for (int f = 0; f < NSF_NUM_FIELDS; ++f) nf += (fieldMask >> f) & 1u;
    if (!nf) return;
    std::vector<double> all(nf * nNodesTotal);
    check(nsf_download(handle_, fieldMask, all.data()), handle_, "nsf_download");
    Array3D_d* dst[NSF_NUM_FIELDS] = {&conservedVariables.rho,  &conservedVariables.rho_u, &conservedVariables.rho_v,
                                      &conservedVariables.rho_w, &conservedVariables.rho_E, &primitiveVariables.u,
                                      &primitiveVariables.v,     &primitiveVariables.w,     &primitiveVariables.p,
                                      &primitiveVariables.T,     &transportProperties.mu,   &transportProperties.kappa};
    size_t q = 0;
    for (int f = 0; f < NSF_NUM_FIELDS; ++f)
      if ((fieldMask >> f) & 1u) {
        dst[f]->data.assign(all.begin() + q * nNodesTotal, all.begin() + (q + 1) * nNodesTotal);
        ++q;
      }
  }

  // Host data of field f (NSF_RHO..NSF_KAPPA) in the mirrors, or nullptr if it was never downloaded.
  const double* mirror(int f) const {
    const Array3D_d* src[NSF_NUM_FIELDS] = {
        &conservedVariables.rho, &conservedVariables.rho_u, &conservedVariables.rho_v, &conservedVariables.rho_w,
        &conservedVariables.rho_E, &primitiveVariables.u, &primitiveVariables.v, &primitiveVariables.w,
        &primitiveVariables.p, &primitiveVariables.T, &transportProperties.mu, &transportProperties.kappa};
    return src[f]->data.size() == nNodesTotal ? src[f]->data.data() : nullptr;
  }

  nsf_solver* handle() const { return handle_; }

 private:
  friend class Solver;
  void bind(nsf_solver* h, const nsf_config& c) {
    handle_ = h;
    NI = size_t(c.NI);
    NJ = size_t(c.NJ);
    NK = size_t(c.NK);
    nNodesTotal = NI * NJ * NK;
    double g[6];
    check(nsf_get_geometry(h, g), h, "nsf_get_geometry");
    const double d[3] = {g[0], g[1], g[2]}, off[3] = {g[3], g[4], g[5]};
    dx = d[0];
    dy = d[1];
    dz = d[2];
    positionOffset = Vector3_d{off[0], off[1], off[2]};
    for (Array3D_d* a : {&conservedVariables.rho, &conservedVariables.rho_u, &conservedVariables.rho_v,
                         &conservedVariables.rho_w, &conservedVariables.rho_E, &primitiveVariables.u,
                         &primitiveVariables.v, &primitiveVariables.w, &primitiveVariables.p, &primitiveVariables.T,
                         &transportProperties.mu, &transportProperties.kappa}) {
      a->NI = NI;
      a->NJ = NJ;
      a->NK = NK;
    }
    nodeTypes.resize(nNodesTotal);
    check(nsf_get_node_types(h, nodeTypes.data()), h, "nsf_get_node_types");
  }
  nsf_solver* handle_ = nullptr;
};

// Solver (src/Solver.h:17-81): owns the device solver; marchTimeStep advances one RK4 step.
class Solver {
 public:
  explicit Solver(const ConfigSettings& p, int device = 0) : params(p), device_(device) {}
  Solver(const Solver&) = delete;
  Solver& operator=(const Solver&) = delete;
  ~Solver() {
    if (h_) nsf_destroy(h_);
  }

  // Solver::initialize (Solver.cpp:22-28).
  void initialize() {
    check(nsf_create(&params.raw, device_, &h_), h_, "nsf_create");
    check(nsf_initialize(h_), h_, "nsf_initialize");
    mesh.bind(h_, params.raw);
    if (device_ >= 0) {
      double t;
      uint64_t lv;
      check(nsf_get_time(h_, &t, &lv, &dt), h_, "nsf_get_time");
    }
  }

  // Solver::marchTimeStep (Solver.cpp:130-167): one step; t, timeLevel and dt as the reference leaves them.
  void marchTimeStep(double& t, ulong& timeLevel) {
    check(nsf_march(h_, 1), h_, "nsf_march");
    uint64_t lv = 0;
    check(nsf_get_time(h_, &t, &lv, &dt), h_, "nsf_get_time");
    timeLevel = ulong(lv);
  }

  // Solver::getConvergenceHistory (Solver.h:27): the recorded change norms (entries not recorded under
  // the ConvHistory setting are absent, as in the reference's vectors).
  const ConservedVariablesVectorGroup& getConvergenceHistory() const {
    uint64_t avail = 0;
    check(nsf_get_history(h_, 0, 0, nullptr, &avail), h_, "nsf_get_history");
    std::vector<double> rows(7 * avail);
    if (avail) check(nsf_get_history(h_, 0, avail, rows.data(), &avail), h_, "nsf_get_history");
    history_ = ConservedVariablesVectorGroup{};
    std::vector<double>* v[5] = {&history_.rho, &history_.rho_u, &history_.rho_v, &history_.rho_w, &history_.rho_E};
    for (uint64_t r = 0; r < avail; ++r)
      for (int f = 0; f < 5; ++f)
        if (rows[7 * r + 2 + f] >= 0) v[f]->push_back(rows[7 * r + 2 + f]);
    return history_;
  }

  nsf_solver* handle() const { return h_; }

  const ConfigSettings params;
  Mesh mesh;
  double dt = 0;

 private:
  int device_;
  nsf_solver* h_ = nullptr;
  mutable ConservedVariablesVectorGroup history_;
};

// Snapshot writer behind OutputManager: each snapshot is downloaded with nsf_download_async into one of two
// page-locked host buffers and written by a worker thread once it has landed, so the solver marches on while
// the snapshot crosses to the host and is formatted. The main thread blocks only when both buffers are still
// owned by snapshots that are in flight or being written.
class SnapshotWriter {
 public:
  // Receives the downloaded fields: fields[f] holds field f (NSF_RHO..NSF_KAPPA) for every node, or is
  // nullptr if f was not asked for.
  using WriteFn = std::function<void(const double* const* fields)>;

  SnapshotWriter() = default;
  SnapshotWriter(const SnapshotWriter&) = delete;
  SnapshotWriter& operator=(const SnapshotWriter&) = delete;
  ~SnapshotWriter() {
    try {
      finish();
    } catch (...) {
    }
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    if (worker_.joinable()) worker_.join();
    for (Buffer& b : bufs_)
      if (b.host) nsf_host_free(b.host);
  }

  // Queue the fields in `fieldMask` of the solution `h` holds now (behind the steps already marched), to
  // be passed to `write` once they are on the host. A mask of 0 calls `write` with no fields.
  void submit(nsf_solver* h, uint32_t fieldMask, size_t nNodes, WriteFn write) {
    fieldMask &= (1u << NSF_NUM_FIELDS) - 1;
    Job job;
    job.h = h;
    job.write = std::move(write);
    size_t nf = 0;
    for (int f = 0; f < NSF_NUM_FIELDS; ++f) job.slot[f] = (fieldMask >> f) & 1u ? int(nf++) : -1;
    job.nNodes = nNodes;
    if (nf) {
      std::unique_lock<std::mutex> lk(mu_);
      const int b = next_;
      next_ ^= 1;
      cv_.wait(lk, [&] { return !bufs_[b].busy; });
      rethrow_locked();
      lk.unlock();
      Buffer& buf = bufs_[b];
      const size_t bytes = nf * nNodes * sizeof(double);
      if (buf.bytes < bytes) {
        if (buf.host) nsf_host_free(buf.host);
        buf.host = nullptr;
        buf.bytes = 0;
        void* p = nullptr;
        check(nsf_host_alloc(bytes, &p), nullptr, "nsf_host_alloc");
        buf.host = static_cast<double*>(p);
        buf.bytes = bytes;
      }
      check(nsf_download_async(h, fieldMask, buf.host, &job.ticket), h, "nsf_download_async");
      job.buffer = b;
      lk.lock();
      buf.busy = true;
    }
    std::lock_guard<std::mutex> lk(mu_);
    jobs_.push_back(std::move(job));
    ++pending_;
    if (!worker_.joinable()) worker_ = std::thread([this] { run(); });
    cv_.notify_all();
  }

  // Wait until every queued snapshot is written; rethrows the first error of a download or a write.
  void finish() {
    std::unique_lock<std::mutex> lk(mu_);
    cv_.wait(lk, [&] { return pending_ == 0; });
    rethrow_locked();
  }

 private:
  struct Buffer {
    double* host = nullptr;
    size_t bytes = 0;
    bool busy = false;
  };
  struct Job {
    nsf_solver* h = nullptr;
    uint64_t ticket = 0;  // 0: nothing downloaded
    int buffer = -1;
    int slot[NSF_NUM_FIELDS];
    size_t nNodes = 0;
    WriteFn write;
  };

  void rethrow_locked() {
    if (error_) {
      std::exception_ptr e = error_;
      error_ = nullptr;
      std::rethrow_exception(e);
    }
  }

  void run() {
    for (;;) {
      Job job;
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return stop_ || !jobs_.empty(); });
        if (jobs_.empty()) return;
        job = std::move(jobs_.front());
        jobs_.pop_front();
      }
      std::exception_ptr err;
      try {
        const double* fields[NSF_NUM_FIELDS] = {};
        if (job.ticket) {
          const nsf_status st = nsf_download_wait(job.h, job.ticket);
          if (st != NSF_OK) throw Error(st, std::string("nsf_download_wait: ") + status_name(st));
          for (int f = 0; f < NSF_NUM_FIELDS; ++f)
            if (job.slot[f] >= 0) fields[f] = bufs_[job.buffer].host + size_t(job.slot[f]) * job.nNodes;
        }
        job.write(fields);
      } catch (...) {
        err = std::current_exception();
      }
      {
        std::lock_guard<std::mutex> lk(mu_);
        if (err && !error_) error_ = err;
        if (job.buffer >= 0) bufs_[job.buffer].busy = false;
        --pending_;
      }
      cv_.notify_all();
    }
  }

  Buffer bufs_[2];
  int next_ = 0;
  std::deque<Job> jobs_;
  size_t pending_ = 0;
  bool stop_ = false;
  std::exception_ptr error_;
  std::mutex mu_;
  std::condition_variable cv_;
  std::thread worker_;
};

// OutputManager (src/OutputManager.h:19-73): ASCII legacy VTK snapshots (i fastest), times.dat,
// norm_*.dat and the status report, in the reference's formats. `dir` replaces the hard-coded ./output.
class OutputManager {
 public:
  explicit OutputManager(const ConfigSettings& p, std::string dir = "output") : params(p), dir_(std::move(dir)) {}

  // OutputManager::initialize (OutputManager.cpp:18-47): create the folder, delete old results except
  // ParaView state files.
  void initialize() {
    namespace fs = std::filesystem;
    fs::path out(dir_);
    if (!(fs::exists(out) && fs::is_directory(out)) && !fs::create_directory(out)) {
      std::cerr << "Output folder could not be created.\n";
      return;
    }
    std::vector<fs::path> old;
    for (const fs::directory_entry& e : fs::recursive_directory_iterator(out))
      if (e.path().generic_string().find(".pvsm") == std::string::npos) old.push_back(e.path());
    for (const fs::path& p : old) {
      std::error_code ec;
      fs::remove(p, ec);
    }
    wallClock_ = std::chrono::steady_clock::now();
    statusClock_ = wallClock_;
  }

  void processInitialOutput(const Mesh& mesh, double t) {  // :51-55
    if (params.saveIC) storeCurrentSolution(mesh, t);
  }

  void processIntermediateOutput(const Mesh& mesh, double t, ulong timeLevel, double dt) {  // :60-83
    if (params.saveIntervals) {
      const bool withinRelevantTimeRegime =
          t >= params.saveIntervalsStartTime && (t <= params.saveIntervalsEndTime || params.saveIntervalsEndTime <= 0);
      bool enoughTimeSinceSave = true;
      if (params.savePeriod > 0) enoughTimeSinceSave = std::fmod(t, params.savePeriod) + dt >= params.savePeriod;
      if (withinRelevantTimeRegime && enoughTimeSinceSave) storeCurrentSolution(mesh, t);
    }
    if (seconds(statusClock_) >= params.statusReportInterval) {
      writeStatusReport_toScreen(t, timeLevel, dt);
      statusClock_ = std::chrono::steady_clock::now();
    }
  }

  void processFinalOutput(const Mesh& mesh, double t, ulong timeLevel, double dt,
                          const ConservedVariablesVectorGroup& convergenceHistory) {  // :86-97
    if (params.saveFinal) storeCurrentSolution(mesh, t);
    writer_.finish();
    writeStatusReport_toScreen(t, timeLevel, dt);
    writeOutputTimes();
    writeConvergenceHistoryFiles(convergenceHistory);
  }

  // The VTK text of the current solution (storeCurrentSolution_vtk, :268-284) from the Mesh's host mirrors
  // (Mesh::syncFromDevice), written to `os`.
  void writeVtk(const Mesh& mesh, double t, std::ostream& os) const {
    const double* fields[NSF_NUM_FIELDS];
    for (int f = 0; f < NSF_NUM_FIELDS; ++f) fields[f] = mesh.mirror(f);
    writeVtkFields(mesh, t, fields, os);
  }

  // The same text from field arrays: fields[f] holds field f (NSF_RHO..NSF_KAPPA) for every node, k fastest;
  // only the fields the settings save are read.
  void writeVtkFields(const Mesh& mesh, double t, const double* const* fields, std::ostream& os) const {
    const uint32_t need = savedFieldMask();
    for (int f = 0; f < NSF_NUM_FIELDS; ++f)
      if ((need >> f) & 1u && !fields[f])
        throw std::logic_error("writeVtk: field " + std::to_string(f) + " is not on the host");
    const size_t sj = mesh.NK, si = mesh.NJ * mesh.NK;
    os << "# vtk DataFile Version 5.1\n";
    os << "Output at time t = " + std::to_string(t) + "\n";
    os << "ASCII\n";
    os << "DATASET STRUCTURED_POINTS\n";
    os << "DIMENSIONS " + std::to_string(mesh.NI) + " " + std::to_string(mesh.NJ) + " " + std::to_string(mesh.NK) + "\n";
    os << "ORIGIN " + std::to_string(-mesh.positionOffset.x * mesh.dx) + " " +
              std::to_string(-mesh.positionOffset.y * mesh.dy) + " " + std::to_string(-mesh.positionOffset.z * mesh.dz) +
              "\n";
    os << "SPACING " + std::to_string(mesh.dx) + " " + std::to_string(mesh.dy) + " " + std::to_string(mesh.dz) + "\n";
    os << "POINT_DATA " + std::to_string(mesh.nNodesTotal) + "\n";
    // Node flags (writeVtkNodeFlags, :125-150): solid ghost 3, solid inactive 4.
    os << "SCALARS Node_Flag int 1\n";
    os << "LOOKUP_TABLE default\n";
    static const int flag[5] = {0, 1, 2, 4, 3};
    for (size_t k = 0; k < mesh.NK; ++k)
      for (size_t j = 0; j < mesh.NJ; ++j)
        for (size_t i = 0; i < mesh.NI; ++i) os << flag[int(mesh.nodeType(i, j, k))] << "\n";
    // Scalars (writeVtkScalarData, :196-211) and vectors (writeVtkVectorData, :246-263).
    const int sc[6] = {NSF_RHO, NSF_RHO_E, NSF_P, NSF_T, NSF_MU, NSF_KAPPA};
    const bool scOn[6] = {params.saveDensity,     params.saveEnergy,    params.savePressure,
                          params.saveTemperature, params.saveViscosity, params.saveThermalCond};
    const char* scName[6] = {"Density",     "Total_Specific_Energy_per_Volume", "Pressure",
                             "Temperature", "Dynamic_Viscosity",                "Thermal_Conductivity"};
    for (int q = 0; q < 6; ++q) {
      if (!scOn[q]) continue;
      const double* v = fields[sc[q]];
      os << "SCALARS " << scName[q] << " double 1\n";
      os << "LOOKUP_TABLE default\n";
      for (size_t k = 0; k < mesh.NK; ++k)
        for (size_t j = 0; j < mesh.NJ; ++j)
          for (size_t i = 0; i < mesh.NI; ++i) os << v[i * si + j * sj + k] << "\n";
    }
    const int vec[2] = {NSF_RHO_U, NSF_U};
    const bool vecOn[2] = {params.saveMomentum, params.saveVelocity};
    const char* vecName[2] = {"Momentum_Density", "Velocity"};
    for (int q = 0; q < 2; ++q) {
      if (!vecOn[q]) continue;
      const double *x = fields[vec[q]], *y = fields[vec[q] + 1], *z = fields[vec[q] + 2];
      os << "VECTORS " << vecName[q] << " double\n";
      for (size_t k = 0; k < mesh.NK; ++k)
        for (size_t j = 0; j < mesh.NJ; ++j)
          for (size_t i = 0; i < mesh.NI; ++i) {
            const size_t n = i * si + j * sj + k;
            os << x[n] << " " << y[n] << " " << z[n] << "\n";
          }
    }
  }

  // Fields a snapshot writes (bit f = NSF_RHO..NSF_KAPPA), from the save* settings.
  uint32_t savedFieldMask() const {
    uint32_t m = 0;
    if (params.saveDensity) m |= 1u << NSF_RHO;
    if (params.saveMomentum) m |= 7u << NSF_RHO_U;
    if (params.saveEnergy) m |= 1u << NSF_RHO_E;
    if (params.saveVelocity) m |= 7u << NSF_U;
    if (params.savePressure) m |= 1u << NSF_P;
    if (params.saveTemperature) m |= 1u << NSF_T;
    if (params.saveViscosity) m |= 1u << NSF_MU;
    if (params.saveThermalCond) m |= 1u << NSF_KAPPA;
    return m;
  }

  // Wait until every snapshot queued so far is on disk (processFinalOutput does this).
  void finishWrites() { writer_.finish(); }

  uint32_t savedSolutions = 0;
  std::vector<double> outputTimes;

 private:
  static double seconds(std::chrono::steady_clock::time_point since) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - since).count();
  }

  // :101-106. The saved fields of the current solution are queued for download and the file is written by
  // the snapshot writer once they have landed; `mesh` must outlive the write (finishWrites).
  void storeCurrentSolution(const Mesh& mesh, double t) {
    const std::string filename = dir_ + "/out.vtk." + std::to_string(savedSolutions);
    auto f = std::make_shared<std::ofstream>(filename);
    if (!*f) {
      std::cout << "Could not open file:  " + filename << std::endl << "Solution was not saved." << std::endl;
      return;
    }
    ++savedSolutions;
    outputTimes.push_back(t);
    const Mesh* m = &mesh;
    writer_.submit(mesh.handle(), savedFieldMask(), mesh.nNodesTotal, [this, m, t, f](const double* const* fields) {
      writeVtkFields(*m, t, fields, *f);
      f->close();
    });
  }

  void writeStatusReport_toScreen(double t, ulong timeLevel, double dt) {  // :289-311
    std::cout << "Simulated time: t = " << t;
    if (params.stopCriterion == StopCriterionEnum::end_time) {
      const double pct = t / params.t_end * 100.;
      std::cout << " , t_end = " << params.t_end << " ( " << std::setprecision(3) << pct << std::setprecision(6)
                << " % )" << std::endl;
    } else {
      std::cout << std::endl;
    }
    std::cout << "Time level: n = " << timeLevel;
    if (params.stopCriterion == StopCriterionEnum::timesteps) {
      const double pct = double(timeLevel) / double(params.stopTimeLevel) * 100.;
      std::cout << " , n_max = " << params.stopTimeLevel << " ( " << std::setprecision(3) << pct
                << std::setprecision(6) << " % )" << std::endl;
    } else {
      std::cout << std::endl;
    }
    std::cout << "Timestep size: dt = " << dt << std::endl;
    std::cout << "Wall clock time: " << std::setprecision(3) << seconds(wallClock_) << std::setprecision(6) << " sec"
              << std::endl
              << std::endl;
  }

  void writeOutputTimes() {  // :314-328
    std::ofstream f(dir_ + "/times.dat");
    if (!f) return;
    for (double time : outputTimes) f << time << std::endl;
  }

  void writeConvergenceHistoryFiles(const ConservedVariablesVectorGroup& h) {  // :331-362
    std::vector<const std::vector<double>*> v;
    std::vector<std::string> names;
    if (params.saveConvergenceHistory != ConvHistoryEnum::none) {
      v.push_back(&h.rho);
      names.push_back("rho");
    }
    if (params.saveConvergenceHistory == ConvHistoryEnum::all) {
      v.insert(v.end(), {&h.rho_u, &h.rho_v, &h.rho_w, &h.rho_E});
      names.insert(names.end(), {"rho_u", "rho_v", "rho_w", "rho_E"});
    }
    for (size_t q = 0; q < names.size(); ++q) {
      std::ofstream f(dir_ + "/norm_" + names[q] + ".dat");
      if (!f) continue;
      for (double n : *v[q]) f << n << std::endl;
    }
  }

  const ConfigSettings params;
  std::string dir_;
  std::chrono::steady_clock::time_point wallClock_ = std::chrono::steady_clock::now(), statusClock_ = wallClock_;
  SnapshotWriter writer_;  // last: its pending writes finish before the members they read are destroyed
};

// Simulation (src/Simulation.h:18-35): initialise, march until the stopping criterion, write output.
class Simulation {
 public:
  explicit Simulation(const ConfigSettings& p, int device = 0, std::string outputDir = "output")
      : params(p), solver(p, device), output(p, std::move(outputDir)) {}

  void run() {  // Simulation.cpp:19-30
    solver.initialize();
    output.initialize();
    output.processInitialOutput(solver.mesh, t);
    while (!checkStoppingCriterion()) {
      solver.marchTimeStep(t, timeLevel);
      output.processIntermediateOutput(solver.mesh, t, timeLevel, solver.dt);
    }
    output.processFinalOutput(solver.mesh, t, timeLevel, solver.dt, solver.getConvergenceHistory());
  }

  const ConfigSettings params;
  Solver solver;
  OutputManager output;
  double t = 0;
  ulong timeLevel = 0;

 private:
  bool checkStoppingCriterion() const {  // Simulation.cpp:34-52
    if (params.stopCriterion == StopCriterionEnum::timesteps) return !(timeLevel < params.stopTimeLevel);
    return !(t < params.t_end);
  }
};

}  // namespace nsfsi
#endif
