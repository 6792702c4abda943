// Device-side pieces of the x-slab decomposition (nsf_slab.cu), used by the slab-group driver (nsf_slab.cpp).
#ifndef NSF_SLAB_H
#define NSF_SLAB_H

#include "nsf_device.cuh"

namespace nsf {

// What a plane transfer moves: the stage output (five conserved fields, every stage) or the filtered
// density of the global density filter (filter steps only).
enum SlabWhat { SLAB_STAGE = 0, SLAB_FILTER = 1 };

// One side of a plane transfer: the slab's grid (device), its local plane, the staging buffer (sI doubles
// per field).
struct SlabTask {
  const Grid* grid;
  int plane;
  int which;
  double* buf;
};

// dir 0: pack the tasks' planes into their buffers; dir 1: unpack buffers into planes. planeWords: the
// largest sI of the tasks' grids.
void launch_slab_copy(const SlabTask* tasks, int ntasks, long long planeWords, int s, int dir, void* stream);
// part[9 g ..]: grid g's four dt maxima and five change-norm sums.
void launch_slab_partials(const Grid* grids, int n, double* part, void* stream);
// out[0..3]: the dt maxima over all slabs, out[4..8]: the change-norm sums in slab order; slab p's partials
// at part[9 at[p] ..].
void launch_slab_combine(const double* part, const int* at, int P, double* out, void* stream);
// The end of step of every grid from those global quantities.
void launch_slab_finalize(Grid* grids, int n, const double* in, void* stream);

}  // namespace nsf
#endif
