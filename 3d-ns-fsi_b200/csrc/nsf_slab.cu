// Kernels of the x-slab decomposition of one grid (nsf_slab.cpp): plane exchanges between slabs and the
// step's global reductions.
//
// A slab holds a contiguous range of the grid's i-planes plus one plane on each side: a halo (a copy of the
// neighbouring slab's plane) or, at the ends, the grid's own x face. Planes are contiguous in the k-fastest,
// i-slowest layout (one plane = sI doubles per field), so an exchange moves whole planes. Which physical
// buffer holds a stage's output rotates from step to step on the device (StepCtl), so the pack and unpack
// kernels read the buffer of each field from the slab's control block at run time, and the transfers
// between them use fixed staging buffers -- one CUDA graph serves every step.
#include <cuda_runtime.h>

#include "nsf_device.cuh"
#include "nsf_internal.h"
#include "nsf_physics.cuh"
#include "nsf_slab.h"

namespace nsf {
namespace {

// The fields a transfer moves: the stage output (five conserved fields), or the filtered density of the
// global density filter (only on filter steps).
__device__ __forceinline__ int slab_fields(const StepCtl* c, int which) { return which == SLAB_STAGE ? 5 : 1; }
__device__ __forceinline__ double* slab_field(const StepCtl* c, int which, int s, int f) {
  return which == SLAB_STAGE ? c->O[s][f] : c->gfDst;
}

// dir 0: plane -> staging buffer (pack); dir 1: staging buffer -> plane (unpack). blockIdx.y = task.
__global__ void k_slab_copy(const SlabTask* __restrict__ tasks, int s, int dir) {
  const SlabTask t = tasks[blockIdx.y];
  const Grid& G = *t.grid;
  const StepCtl* c = G.ctl;
  if (!c->active) return;
  if (t.which == SLAB_FILTER && !c->filterNow) return;
  const int nf = slab_fields(c, t.which);
  const long long plane = G.sI;
  for (int f = 0; f < nf; ++f) {
    double* field = slab_field(c, t.which, s, f) + (long long)t.plane * plane;
    double* buf = t.buf + f * plane;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < plane; q += (long long)gridDim.x * blockDim.x) {
      if (dir == 0)
        buf[q] = field[q];
      else
        field[q] = buf[q];
    }
  }
}

// Each slab of this process: part[9 g .. 9 g + 8] = its four dt maxima (c + |u|, c + |v|, c + |w|, the
// viscous term) and its five change-norm sums (its partial slots in order). One block.
__global__ void k_slab_partials(const Grid* __restrict__ grids, int n, double* __restrict__ part) {
  __shared__ double red[5 * 32];
  __shared__ double tot[5];
  for (int g = 0; g < n; ++g) {
    const Grid& G = grids[g];
    double s[5] = {0, 0, 0, 0, 0};
    for (int q = threadIdx.x; q < G.nNormSlots; q += blockDim.x)
      for (int f = 0; f < 5; ++f) s[f] += G.normPart[5 * q + f];
    flush_norms(tot, s, red);
    if (threadIdx.x == 0) {
      for (int q = 0; q < 4; ++q) part[9 * g + q] = __longlong_as_double(static_cast<long long>(G.ctl->mx[q]));
      for (int f = 0; f < 5; ++f) part[9 * g + 4 + f] = tot[f];
    }
    __syncthreads();
  }
}

// The step's global quantities from every slab's partials (slab p's at part[9 at[p]]): out[0..3] the
// largest dt maxima, out[4..8] the change-norm sums, slabs in order -- the same arithmetic whichever
// process holds which slab. One thread.
__global__ void k_slab_combine(const double* __restrict__ part, const int* __restrict__ at, int P,
                               double* __restrict__ out) {
  if (threadIdx.x != 0) return;
  double mx[4] = {0, 0, 0, 0};
  double sum[5] = {0, 0, 0, 0, 0};
  for (int p = 0; p < P; ++p) {
    const double* v = part + 9 * (long long)at[p];
    for (int q = 0; q < 4; ++q) mx[q] = fmax(mx[q], v[q]);
    for (int f = 0; f < 5; ++f) sum[f] += v[4 + f];
  }
  for (int q = 0; q < 4; ++q) out[q] = mx[q];
  for (int f = 0; f < 5; ++f) out[4 + f] = sum[f];
}

// End of step for every slab from the global quantities (finalize_grid's arithmetic): next dt, t, level,
// history row -- the same values in every slab's control block.
__global__ void k_slab_finalize(Grid* grids, int n, const double* __restrict__ in) {
  if (threadIdx.x != 0) return;
  for (int g = 0; g < n; ++g) {
    Grid* gp = grids + g;
    StepCtl* c = gp->ctl;
    if (!c->active) continue;
    const Consts& C = gp->C;
    const double conv = C.convLim / (in[0] / C.dx + in[1] / C.dy + in[2] / C.dz);
    const double dx2 = C.dx * C.dx, dy2 = C.dy * C.dy, dz2 = C.dz * C.dz;
    const double visc = C.viscLim / (in[3] * (1 / dx2 + 1 / dy2 + 1 / dz2));
    const double tNew = c->t + c->dtUsed;
    double dt = (visc < conv) ? visc : conv;
    if (C.endTime && tNew + dt > C.tEnd) dt = C.tEnd - tNew;
    double* h = gp->hist + 7 * (c->level % MAX_HIST);
    h[0] = tNew;
    h[1] = c->dtUsed;
    for (int f = 0; f < 5; ++f) {
      const bool kept = (f == 0 && C.convHistory != 0) || C.convHistory == 2;
      h[2 + f] = kept ? sqrt(C.dxdydz * in[4 + f]) : -1.0;
    }
    c->t = tNew;
    c->dt = dt;
    c->level += 1;
  }
}

}  // namespace

void launch_slab_copy(const SlabTask* tasks, int ntasks, long long planeWords, int s, int dir, void* stream) {
  if (ntasks <= 0) return;
  const long long b = (planeWords + 255) / 256;
  k_slab_copy<<<dim3(unsigned(b < 256 ? b : 256), unsigned(ntasks)), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      tasks, s, dir);
}

void launch_slab_partials(const Grid* grids, int n, double* part, void* stream) {
  k_slab_partials<<<1, 256, 0, static_cast<cudaStream_t>(stream)>>>(grids, n, part);
}

void launch_slab_combine(const double* part, const int* at, int P, double* out, void* stream) {
  k_slab_combine<<<1, 32, 0, static_cast<cudaStream_t>(stream)>>>(part, at, P, out);
}

void launch_slab_finalize(Grid* grids, int n, const double* in, void* stream) {
  k_slab_finalize<<<1, 32, 0, static_cast<cudaStream_t>(stream)>>>(grids, n, in);
}

}  // namespace nsf
