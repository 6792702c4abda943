// Test program: writes the VTK snapshot of given field values through nsfsi_host.hpp's OutputManager.
// The node types and geometry come from a host-only solver handle (no GPU); the twelve fields are read
// from a raw file (12 x N doubles, reference layout), so the text can be compared byte for byte with what
// the reference's own OutputManager wrote for the same values.
//
//     vtk_check <case.cfg> <fields.bin> <t> <out.vtk>
#include <cstdio>
#include <fstream>
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
  std::ofstream os(argv[4]);
  out.writeVtk(mesh, std::atof(argv[3]), os);
  return os ? 0 : 5;
}
