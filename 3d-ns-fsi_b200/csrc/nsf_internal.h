// Internal declarations shared by the host setup (nsf_setup.cpp), the C ABI (nsf_capi.cpp) and the
// CUDA kernels (nsf_kernels.cu). Not part of the public interface.
#ifndef NSF_INTERNAL_H
#define NSF_INTERNAL_H

#include <cstddef>
#include <cstdint>
#include <map>
#include <string>
#include <vector>

#include "nsfsi.h"

namespace nsf {

// NodeTypeEnum, src/Node.h:27-34 (same values). The device copy of the node-type array also carries
// FILTER_BIT on the fluid nodes that an immersed body filters (ImmersedBoundary::filterNodes).
enum : uint8_t { FLUID_INTERIOR = 0, FLUID_EDGE = 1, FLUID_GHOST = 2, SOLID_INACTIVE = 3, SOLID_GHOST = 4 };
constexpr uint8_t TYPE_MASK = 0x7;
constexpr uint8_t FILTER_BIT = 0x80;
constexpr uint8_t EDGE_PLANE_BIT = 0x40;  // node lies in a mesh-edge boundary's owned box
// Periodic z faces (Grid::zFused): an unfiltered interior fluid node of an interior row at k = 1 (UP) or
// k = NK-2 (DOWN), whose value the stage kernel also writes to its periodic copy at k = NK-1 or k = 0.
constexpr uint8_t ZCOPY_UP_BIT = 0x20;
constexpr uint8_t ZCOPY_DOWN_BIT = 0x10;
// Periodic y faces (Grid::yFused): an unfiltered interior fluid node at j = 1 or j = NJ-2 (the row tells
// which), whose value the stage kernel also writes to its periodic copy at j = NJ-1 or j = 0.
constexpr uint8_t YCOPY_BIT = 0x08;
constexpr int FMETA_LAST = 1 << 30;  // Grid::fmeta: this slot is its node's last
// Edge condition of an x-slab's periodic x face (nsf_slab.cpp): the plane exchange has already copied the
// face's values; the edge item only adds the nodes' stage-4 dt terms, as the whole grid's periodic face does.
constexpr int BC_SLAB_COPY = 16;

struct Box {  // IndexBoundingBox, src/SmallVectors.h:72-104 (inclusive bounds)
  size_t i0, i1, j0, j1, k0, k1;
};

struct EdgeBC {  // one MeshEdgeBoundary: normal axis, side (0 min / 1 max), nsf_bc, owned node box
  int axis, side, bc;
  Box owned;
};

struct GhostRec {  // GhostNode, src/Node.h:15-22
  size_t i, j, k;
  double bi[3], ip[3];
};

struct BodyRec {
  bool sphere;
  double c[3], r;
  int axis;
  std::vector<GhostRec> ghosts;
  std::map<size_t, size_t> ghostIndex;  // node index -> position in ghosts
  std::vector<size_t> filter;
  size_t closureAdded = 0;
};

// Everything the host computes once, before the first step.
struct HostSetup {
  size_t NI = 0, NJ = 0, NK = 0, N = 0;
  double d[3] = {0, 0, 0};    // dx, dy, dz
  double off[3] = {0, 0, 0};  // Mesh::positionOffset
  std::vector<uint8_t> type;  // NodeTypeEnum per node
  std::vector<EdgeBC> edges;  // application order (reverse of the claim order)
  std::vector<BodyRec> bodies;
  // Immersed bodies that act on each other's nodes within a stage (a node in two bodies' lists, a filter
  // stencil or an image-point cell reaching another body's filter node): they must run in the reference's
  // body order, which the fused boundary kernel's dependency levels provide.
  bool bodiesInteract = false;
};

// Setup entry points (nsf_setup.cpp). Return NSF_OK or an error with a message in `err`.
nsf_status build_setup(const nsf_config& cfg, HostSetup& s, std::string& err);
// Initial condition at every node: conserved (5 x N) and primitive/transport (7 x N).
void initial_condition(const nsf_config& cfg, const HostSetup& s, std::vector<double>& cons5,
                       std::vector<double>& prim7);
// Position of node (i,j,k): getNodePosition, src/SmallVectors.h:56-64.
inline void node_position(const HostSetup& s, size_t i, size_t j, size_t k, double p[3]) {
  p[0] = (static_cast<int>(i) - s.off[0]) * s.d[0];
  p[1] = (static_cast<int>(j) - s.off[1]) * s.d[1];
  p[2] = (static_cast<int>(k) - s.off[2]) * s.d[2];
}
// The 8 nodes around a point: getSurroundingNodesBox, src/SmallVectors.h:108-127. Returns false if the
// box would leave the mesh (the reference reads out of range there).
bool surrounding_box(const HostSetup& s, const double p[3], Box& b);
// asIndexList order (z fastest, x slowest), src/SmallVectors.h:89-103.
void box_corners(const HostSetup& s, const Box& b, int64_t out[8]);

}  // namespace nsf

#endif
