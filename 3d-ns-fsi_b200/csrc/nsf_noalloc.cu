// nsf_step_metrics_noalloc: the end-of-step metrics (the five change norms of
// Solver::storeNormsOfChange, Solver.cpp:510-530 / Mesh.cpp:171-178, and the next dt of
// Solver::updateTimeStepSize, Solver.cpp:80-126) for conserved fields that the CALLER holds in device
// memory, computed without allocating anything.
//
// Who needs it: host frameworks that own every byte of device memory and hand this library only
// pointers (a coupling framework or plugin host that forbids third-party cudaMalloc), code running
// while a CUDA stream is being captured into a graph (a cudaMalloc there would not be part of the
// graph and breaks the replay contract), and real-time loops that must not allocate after start-up.
// The solver handle (nsf_create / nsf_march) allocates its scratch; this entry point does not.
//
// Scratch: the per-block partial results of the two-pass reduction live in one file-scope device array
// of kScratchBytes (8 MiB) that every GPU loading this library holds until the process
// exits. One partial (9 doubles) is written per 256 nodes, so grids of up to 29,826,048 nodes fit;
// larger grids are rejected with NSF_ERR_ARG. Every partial the final pass reads is written earlier in
// the same call, so nothing has to be cleared between calls. All calls share the array: two calls whose
// kernels overlap on the GPU (different streams, or different host threads) race on it and must be
// serialised by the caller.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <mutex>

#include "nsf_internal.h"

namespace {

constexpr size_t kScratchBytes = size_t(8) << 20;
constexpr int kTile = 256;  // nodes per partial (threads per block of the first pass)
constexpr int kQ = 9;       // five squared-difference sums, four maxima
constexpr size_t kMaxPartials = kScratchBytes / (kQ * sizeof(double));

__device__ __align__(256) double g_metrics_scratch[kScratchBytes / sizeof(double)];

// Device address of g_metrics_scratch per device, resolved once per device (host code may not use the
// symbol's host-side name as a device address).
double* g_scratch_addr[64] = {};
std::mutex g_scratch_mutex;

struct MetricParams {
  long long NI, NJ, NK, N;
  double gamma, gm1, sc1, re, vmod;
};

__global__ void k_metrics_partial(MetricParams p, const double* __restrict__ old5, const double* __restrict__ new5,
                                  const uint8_t* __restrict__ types, double* __restrict__ partial) {
  __shared__ double red[kQ][kTile / 32];
  const long long n = (long long)blockIdx.x * kTile + threadIdx.x;
  double v[kQ] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  if (n < p.N) {
    const long long i = n / (p.NJ * p.NK), j = n % (p.NJ * p.NK) / p.NK, k = n % p.NK;
    const bool interior = types ? (types[n] & nsf::TYPE_MASK) == nsf::FLUID_INTERIOR
                                : (i > 0 && j > 0 && k > 0 && i < p.NI - 1 && j < p.NJ - 1 && k < p.NK - 1);
    double u[5];
    for (int f = 0; f < 5; ++f) {
      u[f] = new5[f * p.N + n];
      if (interior) {
        const double d = old5[f * p.N + n] - u[f];
        v[f] = d * d;
      }
    }
    const double r1 = 1.0 / (u[0] + 1.0);
    const double uu = u[1] * r1, vv = u[2] * r1, ww = u[3] * r1;
    const double pp = p.gm1 * (u[4] - (u[0] + 1.0) * 0.5 * (uu * uu + vv * vv + ww * ww));
    const double T = (p.gamma * pp - u[0]) * r1;
    const double x = 1.0 + T;
    const double mu = x * sqrt(x) * p.sc1 / (p.re * (T + p.sc1));
    const double c = sqrt((1.0 + p.gamma * pp) / (1.0 + u[0]));
    v[5] = c + fabs(uu);
    v[6] = c + fabs(vv);
    v[7] = c + fabs(ww);
    v[8] = mu / (u[0] + 1.0) * p.vmod;
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int q = 0; q < kQ; ++q) {
    double a = v[q];
    for (int o = 16; o > 0; o >>= 1) {
      const double b = __shfl_xor_sync(0xffffffffu, a, o);
      a = q < 5 ? a + b : fmax(a, b);
    }
    if (lane == 0) red[q][wid] = a;
  }
  __syncthreads();
  if (threadIdx.x < kQ) {
    const int q = threadIdx.x;
    double a = red[q][0];
    for (int w = 1; w < kTile / 32; ++w) a = q < 5 ? a + red[q][w] : fmax(a, red[q][w]);
    partial[(long long)blockIdx.x * kQ + q] = a;
  }
}

// Fixed-order final pass (deterministic): out[0..4] = change norms, out[5] = next dt (min of the convective
// and viscous limits; the end_time clip needs t, which the caller holds, so the caller applies it).
__global__ void k_metrics_final(const double* __restrict__ partial, long long nPartials, double dxdydz, double dx,
                                double dy, double dz, double convLim, double viscLim, double* __restrict__ out) {
  __shared__ double red[kQ][256];
  double v[kQ] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (long long b = threadIdx.x; b < nPartials; b += blockDim.x)
    for (int q = 0; q < kQ; ++q) v[q] = q < 5 ? v[q] + partial[b * kQ + q] : fmax(v[q], partial[b * kQ + q]);
  for (int q = 0; q < kQ; ++q) red[q][threadIdx.x] = v[q];
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s)
      for (int q = 0; q < kQ; ++q)
        red[q][threadIdx.x] = q < 5 ? red[q][threadIdx.x] + red[q][threadIdx.x + s]
                                    : fmax(red[q][threadIdx.x], red[q][threadIdx.x + s]);
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    for (int f = 0; f < 5; ++f) out[f] = sqrt(dxdydz * red[f][0]);
    const double conv = convLim / (red[5][0] / dx + red[6][0] / dy + red[7][0] / dz);
    const double visc = viscLim / (red[8][0] * (1 / (dx * dx) + 1 / (dy * dy) + 1 / (dz * dz)));
    out[5] = (visc < conv) ? visc : conv;
  }
}

}  // namespace

extern "C" nsf_status nsf_step_metrics_noalloc(const nsf_config* cfg, const double* d_old, const double* d_new,
                                               const uint8_t* d_types, double* d_out, void* stream) {
  if (!cfg || !d_old || !d_new || !d_out) return NSF_ERR_ARG;
  const long long NI = (long long)cfg->NI, NJ = (long long)cfg->NJ, NK = (long long)cfg->NK;
  if (NI < 3 || NJ < 3 || NK < 3) return NSF_ERR_ARG;
  const long long N = NI * NJ * NK;
  const long long nPartials = (N + kTile - 1) / kTile;
  if ((unsigned long long)nPartials > kMaxPartials) {
    std::fprintf(stderr,
                 "nsf_step_metrics_noalloc: %lld nodes exceed the fixed 8 MiB scratch (at most %llu nodes)\n", N,
                 (unsigned long long)(kMaxPartials * kTile));
    return NSF_ERR_ARG;
  }
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return NSF_ERR_CUDA;
  double* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_addr[dev]) {
      void* p = nullptr;
      if (cudaGetSymbolAddress(&p, g_metrics_scratch) != cudaSuccess || !p) return NSF_ERR_CUDA;
      g_scratch_addr[dev] = static_cast<double*>(p);
    }
    scratch = g_scratch_addr[dev];
  }
  // Grid spacing by boundary type (Mesh.cpp:44-49), without building a mesh.
  nsf_config c = *cfg;
  if (c.shipped_case) {
    c.bc[0][0] = NSF_BC_INLET;
    c.bc[1][0] = NSF_BC_SYMMETRY;
    c.bc[2][0] = NSF_BC_PERIODIC;
  }
  const long long n3[3] = {NI, NJ, NK};
  const double L[3] = {c.lx, c.ly, c.lz};
  double d[3];
  for (int a = 0; a < 3; ++a) {
    const int t = c.bc[a][0];
    d[a] = L[a] / double(t == NSF_BC_PERIODIC ? n3[a] - 2 : t == NSF_BC_SYMMETRY ? n3[a] - 3 : n3[a] - 1);
  }
  MetricParams p{NI, NJ, NK, N, c.gamma, c.gamma - 1, 1 + c.sutherlands_c2 / c.t0, c.re,
                 std::fmax(4. / 3, c.gamma / c.pr)};
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  k_metrics_partial<<<(unsigned)nPartials, kTile, 0, st>>>(p, d_old, d_new, d_types, scratch);
  k_metrics_final<<<1, 256, 0, st>>>(scratch, nPartials, d[0] * d[1] * d[2], d[0], d[1], d[2],
                                     std::fabs(c.conv_stability_limit), std::fabs(c.visc_stability_limit), d_out);
  return cudaGetLastError() == cudaSuccess ? NSF_OK : NSF_ERR_CUDA;
}
