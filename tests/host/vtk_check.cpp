// Test program: writes the VTK snapshot of given field values through nsfsi_host.hpp's OutputManager.
// The node types and geometry come from a host-only solver handle (no GPU); the twelve fields are read
// from a raw file (12 x N doubles, reference layout), so the text can be compared byte for byte with what
// the reference's own OutputManager wrote for the same values.
//
//     vtk_check <case.cfg> <fields.bin> <t> <out.vtk> [mirrors|packed|writer]
//
// mirrors (default): OutputManager::writeVtk from the Mesh's host mirrors. packed: writeVtkFields from
// pointers to only the fields the settings save (the others null), as the snapshot writer passes them.
// writer: the same write run on SnapshotWriter's worker thread (a job with no download), after checking
// that a job with a download is refused on a handle without a device.
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <vector>

#include "nsfsi_host.hpp"

int main(int argc, char** argv) {
  if (argc < 5) return 2;
  nsfsi::ConfigSettings params(argv[1]);
  if (params.errorOccurred) return 3;
  nsfsi::Solver solver(params, -1);
  solver.initialize();
  nsfsi::Mesh& mesh = solver.mesh;
  const size_t N = mesh.nNodesTotal;
  std::vector<double> all(12 * N);
  std::ifstream in(argv[2], std::ios::binary);
  in.read(reinterpret_cast<char*>(all.data()), std::streamsize(all.size() * sizeof(double)));
  if (!in) return 4;
  nsfsi::Array3D_d* dst[12] = {&mesh.conservedVariables.rho,   &mesh.conservedVariables.rho_u,
                               &mesh.conservedVariables.rho_v, &mesh.conservedVariables.rho_w,
                               &mesh.conservedVariables.rho_E, &mesh.primitiveVariables.u,
                               &mesh.primitiveVariables.v,     &mesh.primitiveVariables.w,
                               &mesh.primitiveVariables.p,     &mesh.primitiveVariables.T,
                               &mesh.transportProperties.mu,   &mesh.transportProperties.kappa};
  for (int f = 0; f < 12; ++f) dst[f]->data.assign(all.begin() + f * N, all.begin() + (f + 1) * N);
  nsfsi::OutputManager out(params, ".");
  const std::string mode = argc > 5 ? argv[5] : "mirrors";
  const double t = std::atof(argv[3]);
  std::ofstream os(argv[4]);
  if (mode == "mirrors") {
    out.writeVtk(mesh, t, os);
    return os ? 0 : 5;
  }
  // only the saved fields, packed as a snapshot download packs them
  const uint32_t mask = out.savedFieldMask();
  std::vector<double> packed;
  for (int f = 0; f < 12; ++f)
    if ((mask >> f) & 1u) packed.insert(packed.end(), all.begin() + f * N, all.begin() + (f + 1) * N);
  const double* fields[12] = {};
  size_t q = 0;
  for (int f = 0; f < 12; ++f)
    if ((mask >> f) & 1u) fields[f] = packed.data() + (q++) * N;
  if (mode == "packed") {
    out.writeVtkFields(mesh, t, fields, os);
    return os ? 0 : 5;
  }
  nsfsi::SnapshotWriter writer;
  try {
    writer.submit(solver.handle(), mask, N, [](const double* const*) {});
    return 6;  // a download needs a device
  } catch (const nsfsi::Error& e) {
    std::cout << "refused: " << nsfsi::status_name(e.status) << std::endl;
  }
  writer.submit(solver.handle(), 0, N, [&](const double* const* none) {
    for (int f = 0; f < 12; ++f)
      if (none[f]) throw std::logic_error("a job without a download got fields");
    out.writeVtkFields(mesh, t, fields, os);
  });
  writer.finish();
  return os ? 0 : 5;
}
