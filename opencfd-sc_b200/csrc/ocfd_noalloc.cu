// ocfd_noalloc.cu -- show_flow_msg over caller-owned device arrays, with no
// device allocation of any kind.
//
// Who needs it.  Every other entry point works on an ocfd_handle, and creating
// one allocates device memory.  Some callers cannot do that: a host solver whose
// device memory all belongs to its own pool allocator (it keeps d,u,v,w,T, f and
// Ajac there and cannot hand out more), or code that runs between kernels on a
// device other streams are using, where cudaFree's implicit device-wide
// synchronisation would stall them.  Such a caller still wants the per-step
// diagnostic of the reference's time loop (show_flow_msg, OCFD_Time_Adv.f90:75-86)
// on its own arrays.  This file gives it that without cudaMalloc, cudaFree or
// any allocating library routine.
//
// How.  The partial sums live in one file-scope static __device__ array of
// fixed size (3 doubles for each of OCFD_NOALLOC_MAX_PLANES partial blocks,
// 96 KiB).  Each k-plane is split into the same number of row bands (more bands
// for thin grids, so that a grid of a few planes still spreads over the SMs);
// one block sums one band in a fixed order and writes its three partials; one
// more block adds the partials in order.  The split depends only on the grid
// size, so two calls on the same arrays give the same bits.  Every slot a call
// reads was written earlier in the same call, so nothing in the array has to
// start at zero and nothing is cleared.
// The first call on a device (with that device current) looks up the array's
// address with cudaGetSymbolAddress and keeps it for the life of the process;
// later calls reuse it.  Because there is one array per device, calls that
// overlap on the same device (two streams, or two host threads) race on it:
// the caller serialises them.
#include <algorithm>
#include <cstdio>
#include <mutex>

#include "ocfd_gpu.h"
#include "ocfd_device.cuh"

namespace {

constexpr int NA_COLS = 32, NA_ROWS = 8;
constexpr int NA_THREADS = NA_COLS * NA_ROWS;
constexpr int NA_MAX_DEVICES = 64;
// partials: 3 per plane; the 3 totals follow at offset 3 * MAX_PLANES
constexpr int NA_SCRATCH_DOUBLES = 3 * OCFD_NOALLOC_MAX_PLANES + 32;

static __device__ __align__(256) double g_noalloc_scratch[NA_SCRATCH_DOUBLES];

std::mutex g_setup_mutex;
double* g_scratch_ptr[NA_MAX_DEVICES] = {};

// fixed-order tree sum over the block; thread 0 ends with the totals
__device__ __forceinline__ void na_block_sum3(double (&v)[3], double* sm) {
  const int t = (int)(threadIdx.y * blockDim.x + threadIdx.x);
  for (int q = 0; q < 3; q++) sm[q * NA_THREADS + t] = v[q];
  __syncthreads();
  for (int s = NA_THREADS / 2; s > 0; s >>= 1) {
    if (t < s)
      for (int q = 0; q < 3; q++) sm[q * NA_THREADS + t] += sm[q * NA_THREADS + t + s];
    __syncthreads();
  }
  for (int q = 0; q < 3; q++) v[q] = sm[q * NA_THREADS];
}

// Row band (blockIdx.x) of k-plane blockIdx.y + 1: sum of f5/J, rho|u|^2/2/J
// and p00 rho^(1-gamma) T/J.  Threads (32, 8): i along x, rows along y.
__global__ void __launch_bounds__(NA_THREADS) k_flow_msg_planes(ocfd::Grid G, double gamma, double ma, int rows,
                                                                const double* f, const double* d, const double* u,
                                                                const double* v, const double* w, const double* T,
                                                                const double* ajac, double* part) {
  __shared__ double sm[3 * NA_THREADS];
  const double p00 = 1.0 / (gamma * ma * ma);
  const double tmp1 = 1.0 - gamma;
  const int k = blockIdx.y + 1;
  const int j0 = blockIdx.x * rows + 1, j1 = min(G.ny, j0 + rows - 1);
  double s[3] = {0.0, 0.0, 0.0};
  for (int j = j0 + (int)threadIdx.y; j <= j1; j += NA_ROWS) {
    for (int i = (int)threadIdx.x + 1; i <= G.nx; i += NA_COLS) {
      const long long c = G.ih(i, j, k);
      const double tmp0 = 1.0 / ajac[c];
      const double dd = d[c], uu = u[c], vv = v[c], ww = w[c];
      s[0] += f[G.ii(i, j, k) + 4 * G.n] * tmp0;
      s[1] += dd * (uu * uu + vv * vv + ww * ww) * 0.5 * tmp0;
      s[2] += p00 * pow(dd, tmp1) * T[c] * tmp0;
    }
  }
  na_block_sum3(s, sm);
  if (threadIdx.x == 0 && threadIdx.y == 0)
    for (int q = 0; q < 3; q++) part[((long long)blockIdx.y * gridDim.x + blockIdx.x) * 3 + q] = s[q];
}

__global__ void __launch_bounds__(NA_THREADS) k_flow_msg_total(const double* part, int nparts, double* out) {
  __shared__ double sm[3 * NA_THREADS];
  double v[3] = {0.0, 0.0, 0.0};
  for (int b = threadIdx.x; b < nparts; b += NA_THREADS)
    for (int q = 0; q < 3; q++) v[q] += part[b * 3 + q];
  na_block_sum3(v, sm);
  if (threadIdx.x == 0)
    for (int q = 0; q < 3; q++) out[q] = v[q];
}

// The array's address on the current device, looked up once per device.
int scratch_for_current_device(double** out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= NA_MAX_DEVICES) return OCFD_E_CUDA;
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_ptr[dev]) {
    double* ptr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress((void**)&ptr, g_noalloc_scratch);
    if (e != cudaSuccess || !ptr) {
      std::fprintf(stderr, "ocfd_show_flow_msg_noalloc: cudaGetSymbolAddress failed on device %d: %s\n", dev,
                   cudaGetErrorString(e));
      return OCFD_E_CUDA;
    }
    g_scratch_ptr[dev] = ptr;
  }
  *out = g_scratch_ptr[dev];
  return OCFD_OK;
}

}  // namespace

extern "C" int ocfd_show_flow_msg_noalloc(const ocfd_params* p, const double* f, const double* const prims[5],
                                          const double* ajac, void* stream, double E0[3]) {
  if (!p || !f || !prims || !ajac || !E0) return OCFD_E_PARAM;
  for (int q = 0; q < 5; q++)
    if (!prims[q]) return OCFD_E_PARAM;
  if (p->nx < 1 || p->ny < 1 || p->nz < 1 || p->lap != ocfd::LAP) return OCFD_E_PARAM;
  if (p->nz > OCFD_NOALLOC_MAX_PLANES) {
    std::fprintf(stderr,
                 "ocfd_show_flow_msg_noalloc: nz = %d exceeds the static scratch limit of %d k-planes; "
                 "use ocfd_gpu_show_flow_msg on a handle instead\n",
                 p->nz, OCFD_NOALLOC_MAX_PLANES);
    return OCFD_E_PARAM;
  }
  cudaStream_t st = (cudaStream_t)stream;
  // the copy to host memory and the wait below cannot be captured
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &cs) != cudaSuccess) return OCFD_E_CUDA;
  if (cs != cudaStreamCaptureStatusNone) return OCFD_E_PARAM;
  double* scratch = nullptr;
  int r = scratch_for_current_device(&scratch);
  if (r) return r;
  ocfd::Grid G;
  G.nx = p->nx;
  G.ny = p->ny;
  G.nz = p->nz;
  G.nxh = p->nx + 2 * ocfd::LAP;
  G.nyh = p->ny + 2 * ocfd::LAP;
  G.nzh = p->nz + 2 * ocfd::LAP;
  G.n = (long long)G.nx * G.ny * G.nz;
  G.nh = (long long)G.nxh * G.nyh * G.nzh;
  double* part = scratch;
  double* total = scratch + 3 * OCFD_NOALLOC_MAX_PLANES;
  // row bands per plane: about four blocks per SM of a B200 over the whole
  // grid, at least 8 rows a band, at most OCFD_NOALLOC_MAX_PLANES bands in all
  int bands = std::min({(G.ny + NA_ROWS - 1) / NA_ROWS, std::max(1, OCFD_NOALLOC_MAX_PLANES / G.nz),
                        std::max(1, (4 * 148 + G.nz - 1) / G.nz)});
  const int rows = (G.ny + bands - 1) / bands;
  bands = (G.ny + rows - 1) / rows;
  k_flow_msg_planes<<<dim3(bands, G.nz), dim3(NA_COLS, NA_ROWS), 0, st>>>(
      G, p->gamma, p->ma, rows, f, prims[0], prims[1], prims[2], prims[3], prims[4], ajac, part);
  k_flow_msg_total<<<1, NA_THREADS, 0, st>>>(part, bands * G.nz, total);
  if (cudaGetLastError() != cudaSuccess) return OCFD_E_CUDA;
  double host[3];
  if (cudaMemcpyAsync(host, total, sizeof(host), cudaMemcpyDeviceToHost, st) != cudaSuccess) return OCFD_E_CUDA;
  if (cudaStreamSynchronize(st) != cudaSuccess) return OCFD_E_CUDA;
  const double N = (double)G.n;
  for (int q = 0; q < 3; q++) E0[q] = host[q] / N;
  return OCFD_OK;
}
