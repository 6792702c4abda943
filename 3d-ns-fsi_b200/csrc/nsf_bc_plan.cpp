// Host-side plan of the fused boundary kernel (k_bc, nsf_kernels.cu): the boundary work of one stage --
// solid-node copies, mesh-edge conditions, near-body filter, ghost interpolation, filter write-back and the
// solid inactive nodes' dt terms -- split into dependency levels. An item's level is one more than the
// level of every item that writes a node it reads (reads of nodes nobody writes in the stage, such as the
// interior nodes the stage kernel computed, are level 0), and it is above the level of every item that
// reads, expecting the old value, a node it overwrites. Items of one level touch disjoint data, so k_bc
// runs a level with all its blocks at once and separates levels with grid barriers; the result equals the
// reference's sequential order (Mesh::applyAllBoundaryConditions, Mesh.cpp:155-167: edges x, y, z, then
// each immersed body's filter and ghosts, Boundary.cpp:427-457).
//
// Periodic copies are followed to the node whose value they finally copy: a y-face node whose periodic
// source lies on a periodic x face reads that x-face node's own source (the copies are exact, so the
// value is the same), which keeps chains of periodic copies in one level.
#include <algorithm>
#include <cstdint>
#include <vector>

#include "nsf_device.cuh"
#include "nsf_internal.h"

namespace nsf {

namespace {

// (i, j, k) inside face e's owned box?
bool in_box(const Grid& G, int e, const int ijk[3]) {
  const int* b = G.eBox[e];
  return ijk[0] >= b[0] && ijk[0] <= b[1] && ijk[1] >= b[2] && ijk[1] <= b[3] && ijk[2] >= b[4] && ijk[2] <= b[5];
}

}  // namespace

// The node a periodic face node finally copies: the face's opposite interior-plane node, followed through
// further periodic faces that own it (at most two more hops: one per other axis). The device edge kernel
// resolves the source the same way (periodic_source in nsf_kernels.cu).
void periodic_source_host(const Grid& G, int axis, int side, int ijk[3]) {
  const int nAx[3] = {G.NI, G.NJ, G.NK};
  ijk[axis] = side == 0 ? nAx[axis] - 2 : 1;
  for (int hop = 0; hop < 2; ++hop) {
    int found = -1;
    for (int e = 0; e < G.nEdge && found < 0; ++e)
      if (G.eBc[e] == NSF_BC_PERIODIC && in_box(G, e, ijk)) found = e;
    if (found < 0) return;
    const int a = G.eAxis[found];
    ijk[a] = G.eSide[found] == 0 ? nAx[a] - 2 : 1;
  }
}

int bc_plan_member(const Grid& G, const std::vector<EdgeBlock> edgeBlocks[3], const BcMemberInput& in,
                   BcMemberLevels& out) {
  const size_t Nd = size_t(G.N);
  // Per node: level of the last item writing all five fields (solid copy, edge condition, ghost) and of the
  // last filter write-back (rho and rho_E only); highest level of an item reading rho / rho_E, and the
  // momenta, from the stage buffer (a later writer must come after it).
  std::vector<int8_t> wA(Nd, 0), wR(Nd, 0), rR(Nd, 0), rM(Nd, 0);
  for (long long n : in.snode) wA[size_t(n)] = 1;  // solid-node copies: level 1
  int levels = in.snode.empty() ? 0 : 1;
  auto dev = [&](const int ijk[3]) { return (long long)ijk[0] * G.sI + (long long)ijk[1] * G.sJ + ijk[2]; };
  // reads of solid nodes off the mesh faces go to the solid copy's source (ld_res; EdgeBlock::solidSrc,
  // Grid::fsolid), so they wait for nothing
  auto solidOff = [&](long long r) {
    const uint8_t t = in.typeDev[size_t(r)], k = t & TYPE_MASK;
    return (k == SOLID_GHOST || k == SOLID_INACTIVE) && !(t & EDGE_PLANE_BIT);
  };
  // (a ghost node stops being one once a body's ghost item has written it: readers of a later body read
  // the ghost value, as the reference's next body does)
  std::vector<uint8_t> ghostDone(Nd, 0);
  auto resolved = [&](long long r) { return solidOff(r) && !ghostDone[size_t(r)]; };
  auto depR = [&](long long r) { return resolved(r) ? 0 : std::max(int(wA[size_t(r)]), int(wR[size_t(r)])); };
  auto depM = [&](long long r) { return resolved(r) ? 0 : int(wA[size_t(r)]); };
  auto readR = [&](long long r, int L) { rR[size_t(r)] = int8_t(std::max(int(rR[size_t(r)]), L)); };
  auto readM = [&](long long r, int L) { rM[size_t(r)] = int8_t(std::max(int(rM[size_t(r)]), L)); };
  // a write of every field at n: after every earlier write and read of it
  auto afterAll = [&](long long n) {
    const size_t q = size_t(n);
    return 1 + std::max({int(wA[q]), int(wR[q]), int(rR[q]), int(rM[q])});
  };
  auto grow = [&](std::vector<std::vector<EdgeBlock>>& v, int L) {
    if (int(v.size()) < L) v.resize(size_t(L));
  };
  auto item = [&](std::vector<std::vector<int>>& v, int L, int q) {
    if (int(v.size()) < L) v.resize(size_t(L));
    v[size_t(L - 1)].push_back(q);
    levels = std::max(levels, L);
  };
  out.edges.clear();
  out.filter.clear();
  out.ghost.clear();
  // mesh-edge conditions, axes in the reference's application order (a face never reads nodes of the other
  // face of its own axis)
  for (int axis = 0; axis < 3; ++axis) {
    std::vector<std::pair<long long, int8_t>> written;
    for (const EdgeBlock& eb : edgeBlocks[axis]) {
      const int* b = G.eBox[eb.e];
      const int ax1 = axis == 0 ? 1 : 0, ax2 = axis == 2 ? 1 : 2;
      const int side = G.eSide[eb.e], bc = G.eBc[eb.e];
      const long long st = axis == 0 ? G.sI : axis == 1 ? G.sJ : 1;
      std::vector<unsigned long long> maskOf;  // per level
      unsigned long long solidSrc = 0;
      for (int ty = 0; ty < kEdgeRows; ++ty)
        for (int tx = 0; tx < 32; ++tx) {
          const int a = eb.a0 + ty, bb = eb.b0 + tx;
          if (a > b[2 * ax1 + 1] || bb > b[2 * ax2 + 1] || !((eb.mask >> (ty * 32 + tx)) & 1)) continue;
          int ijk[3];
          ijk[axis] = b[2 * axis];
          ijk[ax1] = a;
          ijk[ax2] = bb;
          const long long n = dev(ijk);
          std::vector<long long> reads;
          const long long sgn = side == 0 ? 1 : -1;
          if (bc == NSF_BC_INLET) {
            const long long s1 = ax1 == 0 ? G.sI : G.sJ, s2 = ax2 == 1 ? G.sJ : 1;
            std::vector<long long> ms = {n};
            if (a < b[2 * ax1 + 1]) ms.push_back(n + s1);
            if (a > b[2 * ax1]) ms.push_back(n - s1);
            if (bb < b[2 * ax2 + 1]) ms.push_back(n + s2);
            if (bb > b[2 * ax2]) ms.push_back(n - s2);
            for (long long m : ms) {
              reads.push_back(m + sgn * st);
              reads.push_back(m + 2 * sgn * st);
            }
          } else if (bc == NSF_BC_OUTLET) {
            reads.push_back(n + sgn * st);
            reads.push_back(n + 2 * sgn * st);
          } else if (bc == BC_SLAB_COPY) {
            reads.push_back(n);
          } else if (bc == NSF_BC_PERIODIC) {
            int src[3] = {ijk[0], ijk[1], ijk[2]};
            periodic_source_host(G, axis, side, src);
            reads.push_back(dev(src));
          } else {
            reads.push_back(n + 2 * sgn * st);
          }
          int L = afterAll(n);
          for (long long r : reads) {
            if (solidOff(r)) solidSrc |= 1ull << (ty * 32 + tx);
            L = std::max({L, 1 + depR(r), 1 + depM(r)});
          }
          for (long long r : reads) {
            readR(r, L);
            readM(r, L);
          }
          written.push_back({n, int8_t(L)});
          if (int(maskOf.size()) < L) maskOf.resize(size_t(L), 0ull);
          maskOf[size_t(L - 1)] |= 1ull << (ty * 32 + tx);
        }
      for (size_t L = 0; L < maskOf.size(); ++L)
        if (maskOf[L]) {
          grow(out.edges, int(L) + 1);
          EdgeBlock e2 = eb;
          e2.mask = maskOf[L];
          e2.solidSrc = solidSrc & maskOf[L];
          out.edges[L].push_back(e2);
          levels = std::max(levels, int(L) + 1);
        }
    }
    for (auto& w : written) wA[size_t(w.first)] = w.second;  // the next axis reads this axis' results
  }
  // immersed bodies, one after another in the reference's order (Mesh.cpp:164-165): each body's filter
  // (Jacobi: every filtered value from the values before any of that body's write-backs), its write-backs,
  // then its ghosts
  const int nF = int(in.fnode.size()), nG = int(in.gnode.size()), nZ = int(in.inode.size());
  int nBodies = 0;
  for (int b : in.fbody) nBodies = std::max(nBodies, b + 1);
  for (int b : in.gbody) nBodies = std::max(nBodies, b + 1);
  std::vector<int> lf(size_t(nF), 1);
  for (int body = 0; body < nBodies; ++body) {
    for (int f = 0; f < nF; ++f) {
      if (in.fbody[size_t(f)] != body) continue;
      const long long n = in.fnode[size_t(f)];
      const long long nb[7] = {n, n + G.sI, n - G.sI, n + G.sJ, n - G.sJ, n + 1, n - 1};
      int L = 1;
      for (long long r : nb) L = std::max(L, 1 + depR(r));
      // the node's earlier slot wrote fpre / fnew and (stage 4) this slot reads its fpre
      if (in.fidx[size_t(n)] != f) L = std::max(L, 1 + lf[size_t(in.fidx[size_t(n)])]);
      for (long long r : nb) readR(r, L);
      readM(n, L);  // stage 4 reads the node's momenta
      lf[size_t(f)] = L;
      item(out.filter, L, f);
    }
    for (int f = 0; f < nF; ++f) {
      if (in.fbody[size_t(f)] != body) continue;
      const size_t n = size_t(in.fnode[size_t(f)]);
      const int L = std::max({1 + lf[size_t(f)], 1 + int(wA[n]), 1 + int(wR[n]), 1 + int(rR[n])});
      wR[n] = int8_t(L);
      item(out.ghost, L, nG + f);
    }
    for (int q = 0; q < nG; ++q) {
      if (in.gbody[size_t(q)] != body) continue;
      const long long gn = in.gnode[size_t(q)];
      int L = afterAll(gn);
      std::vector<std::pair<long long, bool>> rd;  // corner, reads rho / rho_E from the stage buffer
      for (int m = 0; m < 8; ++m) {
        const long long c = in.gcell[8 * size_t(q) + m];
        if ((in.typeDev[size_t(c)] & TYPE_MASK) == SOLID_GHOST) continue;  // zero weights: not read
        const int src = in.gsrc[8 * size_t(q) + m];
        L = std::max(L, 1 + depM(c));
        if (src >= 0)
          L = std::max(L, 1 + lf[size_t(src)]);
        else
          L = std::max(L, 1 + depR(c));
        rd.push_back({c, src < 0});
      }
      for (auto& r : rd) {
        readM(r.first, L);
        if (r.second) readR(r.first, L);
      }
      wA[size_t(gn)] = int8_t(L);
      item(out.ghost, L, q);
    }
    for (int q = 0; q < nG; ++q)
      if (in.gbody[size_t(q)] == body) ghostDone[size_t(in.gnode[size_t(q)])] = 1;
  }
  // stage-4 dt terms of the solid inactive nodes (their stored values, or their copied conserved values)
  for (int z = 0; z < nZ; ++z) {
    const long long n = in.inode[size_t(z)];
    item(out.ghost, 1 + std::max(depR(n), depM(n)), nG + nF + z);
  }
  out.levels = levels;
  out.solid = (long long)in.snode.size();
  return levels;
}

void bc_flatten(const std::vector<const BcMemberLevels*>& members, BcFlat& out) {
  const int M = int(members.size());
  int levels = 0;
  for (const BcMemberLevels* m : members) levels = std::max(levels, m->levels);
  out.levels = levels;
  out.memberLevels.clear();
  for (const BcMemberLevels* m : members) out.memberLevels.push_back(m->levels);
  out.edges.clear();
  out.items.clear();
  out.edgeStart.assign(size_t(levels) * (M + 1), 0);
  out.itemStart.assign(size_t(levels) * 2 * (M + 1), 0);
  for (int L = 0; L < levels; ++L) {
    for (int g = 0; g < M; ++g) {
      out.edgeStart[size_t(L) * (M + 1) + g] = int(out.edges.size());
      if (L < int(members[g]->edges.size()))
        for (EdgeBlock e : members[g]->edges[size_t(L)]) {
          e.g = g;
          out.edges.push_back(e);
        }
    }
    out.edgeStart[size_t(L) * (M + 1) + M] = int(out.edges.size());
    for (int c = 0; c < 2; ++c) {
      int* start = out.itemStart.data() + (size_t(L) * 2 + c) * (M + 1);
      for (int g = 0; g < M; ++g) {
        start[g] = int(out.items.size());
        const auto& lists = c == 0 ? members[g]->filter : members[g]->ghost;
        if (L < int(lists.size())) out.items.insert(out.items.end(), lists[size_t(L)].begin(), lists[size_t(L)].end());
      }
      start[M] = int(out.items.size());
    }
  }
  // threads one member needs for a level: all its items at once (edge blocks count 64 threads each; the
  // solid-node copies run in the first level)
  long long work = 1;
  out.work.assign(size_t(M), 1);
  for (int L = 0; L < levels; ++L)
    for (int g = 0; g < M; ++g) {
      const size_t eb = size_t(L) * (M + 1) + g, ib = size_t(L) * 2 * (M + 1) + g;
      long long w = 64ll * (out.edgeStart[eb + 1] - out.edgeStart[eb]);
      w += out.itemStart[ib + 1] - out.itemStart[ib];
      w += out.itemStart[ib + M + 2] - out.itemStart[ib + M + 1];
      if (L == 0) w += members[g]->solid;
      work = std::max(work, w);
      out.work[size_t(g)] = std::max(out.work[size_t(g)], w);
    }
  out.maxWork = work;
}

std::vector<int> bc_block_ranges(const BcFlat& fl, int capacity) {
  const int M = int(fl.work.size());
  if (M == 0 || capacity < M) return {};
  std::vector<int> n(static_cast<size_t>(M));
  long long total = 0;
  for (long long w : fl.work) total += w;
  int used = 0;
  for (int g = 0; g < M; ++g) {
    const long long need = (fl.work[size_t(g)] + 255) / 256;
    const long long share = (long long)((double)fl.work[size_t(g)] / double(total) * (capacity - M)) + 1;
    n[size_t(g)] = int(std::max<long long>(1, std::min(need, share)));
    used += n[size_t(g)];
  }
  std::vector<int> start(size_t(M) + 1, 0);
  for (int g = 0; g < M; ++g) start[size_t(g) + 1] = start[size_t(g)] + n[size_t(g)];
  (void)used;
  return start;
}

}  // namespace nsf
