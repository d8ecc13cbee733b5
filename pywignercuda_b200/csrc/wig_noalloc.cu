// Observables of a Wigner function for callers that cannot allocate device
// memory.
//
// The regular path (wig_run) reduces the observables through partial sums in
// scratch that the handle allocates with cudaMalloc.  Some callers cannot
// allocate at all -- for example a custom allocator hook, where a cudaMalloc
// would re-enter the allocator, or a deployment that forbids device allocation
// after start-up.  (Host functions enqueued with cudaLaunchHostFunc are not
// such callers: CUDA forbids any CUDA call inside them, this one included.)
// This entry point
// computes the same 11 observables (the sample wig_run records for a W it does
// not normalise) with its per-row partial sums in a file-scope device array of
// fixed size, so it allocates nothing.
//
// Limits and sharing: grids up to NOALLOC_MAX_ROWS rows (n_p) and 4096 columns
// (n_x).  Every call on a device uses the same array; each call overwrites the
// rows it reads before reading them (nothing has to start at zero), but calls
// whose kernels overlap on the GPU race on the array.  The first call on a
// device looks up the array's device address (cudaGetSymbolAddress) with that
// device current; make that first call before any stream capture.  With CUDA's
// lazy module loading (the default) that first call also loads this module,
// which places the array and the kernels in device memory -- an allocation
// the driver makes -- so make it (a warm-up call on a small W will do) at
// start-up, before allocation is forbidden or an allocator hook is installed.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <mutex>

#include "../../include/wigner_b200.h"
#include "wig_wigner.cuh"

int wig_record_error(int code, const char* msg);   // wig_capi.cu

namespace {

constexpr int NOALLOC_MAX_ROWS = 4096;
constexpr int NOALLOC_MAX_COLS = 4096;
constexpr int NOALLOC_THREADS = 256;
constexpr int NOALLOC_MAX_DEVICES = 64;

// per-row partial sums: [row][wig::NACC] (4096 x 12 doubles = 384 KB per device)
static __device__ __align__(256) double g_noalloc_rows[NOALLOC_MAX_ROWS * wig::NACC];

std::mutex g_noalloc_mu;
double* g_noalloc_ptr[NOALLOC_MAX_DEVICES] = {nullptr};

// Row i of W -> g[i][0..11] (sum Re W, sum Im W and the ten weighted sums).
__global__ void __launch_bounds__(NOALLOC_THREADS)
noalloc_rows(const double2* __restrict__ W, int n_x, const double* __restrict__ x_tab,
             const double* __restrict__ p_tab, const double* __restrict__ dv_tab,
             const double* __restrict__ v0_tab, double mass, double* __restrict__ g) {
  __shared__ double red[NOALLOC_THREADS / 32][wig::NACC];
  double acc[wig::NACC];
#pragma unroll
  for (int v = 0; v < wig::NACC; ++v) acc[v] = 0.;
  const int row = blockIdx.x;
  const double p = p_tab[row];
  const double2* Wr = W + (size_t)row * n_x;
  for (int j = threadIdx.x; j < n_x; j += NOALLOC_THREADS)
    wig::accumulate_obs(acc, Wr[j], x_tab[j], p, dv_tab[j], v0_tab[j], mass);
  wig::block_sum<NOALLOC_THREADS, wig::NACC>(acc, red);
  if (threadIdx.x < wig::NACC) g[(size_t)row * wig::NACC + threadIdx.x] = red[0][threadIdx.x];
}

// One CTA: rows summed in a fixed order, observables written to obs[WIG_NOBS].
__global__ void __launch_bounds__(NOALLOC_THREADS)
noalloc_finish(const double* __restrict__ g, int n_p, double dXdP, double* __restrict__ obs) {
  __shared__ double red[NOALLOC_THREADS / 32][wig::NACC];
  double acc[wig::NACC];
#pragma unroll
  for (int v = 0; v < wig::NACC; ++v) acc[v] = 0.;
  for (int i = threadIdx.x; i < n_p; i += NOALLOC_THREADS) {
#pragma unroll
    for (int v = 0; v < wig::NACC; ++v) acc[v] += g[(size_t)i * wig::NACC + v];
  }
  wig::block_sum<NOALLOC_THREADS, wig::NACC>(acc, red);
  if (threadIdx.x < WIG_NOBS)
    obs[threadIdx.x] = threadIdx.x == 0 ? red[0][0] * dXdP : dXdP * red[0][threadIdx.x + 1];
}

}  // namespace

extern "C" int wig_observables_noalloc(const void* W_dev, int32_t n_x, int32_t n_p, double dx, double dp,
                                       double mass, const double* x_tab, const double* p_tab,
                                       const double* dv_tab, const double* v0_tab, double* obs_dev,
                                       void* stream) {
  char msg[256];
  if (!W_dev || !x_tab || !p_tab || !dv_tab || !v0_tab || !obs_dev)
    return wig_record_error(WIG_ERR_ARG, "wig_observables_noalloc: null pointer argument");
  if (n_x < 1 || n_p < 1 || n_x > NOALLOC_MAX_COLS || n_p > NOALLOC_MAX_ROWS) {
    snprintf(msg, sizeof(msg), "wig_observables_noalloc: grid %d x %d exceeds the static scratch limit of %d "
             "rows x %d columns", n_x, n_p, NOALLOC_MAX_ROWS, NOALLOC_MAX_COLS);
    return wig_record_error(WIG_ERR_ARG, msg);
  }
  if (((uintptr_t)W_dev & 15) != 0)
    return wig_record_error(WIG_ERR_ARG, "wig_observables_noalloc: W must be 16-byte aligned");
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= NOALLOC_MAX_DEVICES)
    return wig_record_error(WIG_ERR_CUDA, "wig_observables_noalloc: no usable current device");
  double* g = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
      // the host-side name of the array is not a device address: look the
      // device address up once per device, with that device current
      void* p = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_rows);
      if (e != cudaSuccess) {
        snprintf(msg, sizeof(msg), "wig_observables_noalloc: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
        return wig_record_error(WIG_ERR_CUDA, msg);
      }
      g_noalloc_ptr[dev] = (double*)p;
    }
    g = g_noalloc_ptr[dev];
  }
  cudaStream_t st = (cudaStream_t)stream;
  noalloc_rows<<<n_p, NOALLOC_THREADS, 0, st>>>((const double2*)W_dev, n_x, x_tab, p_tab, dv_tab, v0_tab, mass, g);
  noalloc_finish<<<1, NOALLOC_THREADS, 0, st>>>(g, n_p, dx * dp, obs_dev);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    snprintf(msg, sizeof(msg), "wig_observables_noalloc: launch: %s", cudaGetErrorString(e));
    return wig_record_error(WIG_ERR_CUDA, msg);
  }
  return WIG_OK;
}
