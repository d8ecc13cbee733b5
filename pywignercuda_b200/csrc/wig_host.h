// Host-side helpers shared by the library's translation units (internal; not
// part of the C ABI): error recording, the NVRTC -> module -> function -> launch
// path of the JIT-compiled kernels, device allocation lists and the FP32
// twiddle rounding.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/wigner_b200.h"

namespace wighost {

extern thread_local std::string g_last_error;

// Record a printf-style message as the thread's last error; returns code.
int fail(int code, const char* fmt, ...);

#define WIG_CUDA(call)                                                                  \
  do {                                                                                  \
    cudaError_t e_ = (call);                                                            \
    if (e_ != cudaSuccess)                                                              \
      return wighost::fail(e_ == cudaErrorMemoryAllocation ? WIG_ERR_NOMEM : WIG_ERR_CUDA, \
                           "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
  } while (0)

// NVRTC source -> sm_100a CUBIN (compile only; no GPU needed).  Takes the JIT lock itself
// when `lock` is set.
int nvrtc_compile_locked(const std::string& src, std::vector<char>* cubin, std::string* log, bool verbose);
// Module of `src` on `device` (compiled once per process and cached).
int get_module(const std::string& src, int device, CUmodule* mod);
int get_fn(CUmodule mod, const char* name, CUfunction* f, int dyn_smem);
int launch(CUfunction f, unsigned grid, unsigned block, unsigned smem, cudaStream_t st, void** args);
int copy_log(const std::string& log, char* out, int64_t cap);
// Blocks that can be resident per SM for a launch shape (1 when the query is unavailable).
int occupancy(CUfunction f, int threads, int dyn_smem);

int launch2d(CUfunction f, unsigned gx, unsigned gy, unsigned block, unsigned smem, cudaStream_t st, void** args);
bool pow2_in_range(int n);                    // power of two in [16, 4096]
int clampi(int v, int lo, int hi);
int round_warp(int v);                        // up to a multiple of 32
// A constant as the reference's kernels see it: '%f' text (or exact), and its value.
std::string fmt_const(double v, int mode);
double kval(double v, int mode);
// numpy linspace(-a, a - 2a/n, n) put through fftshift
std::vector<double> shifted_range(double amp, int n);
// tw[m] = exp(-2 pi i m / n), m < n, extended precision
std::vector<double2> twiddles(int n);
std::string expr_or(const char* s, const char* dflt);
// An expression string that can be pasted between parentheses of a function body.
bool safe_expr(const std::string& e);
extern const char* kMathPrelude;
// Grow a device observable buffer to `need` doubles.
int ensure_obs(double** buf, size_t* cap, size_t need);
// WIG_ERR_NONFINITE unless all n values are finite.
int check_finite(const double* v, size_t n, const char* what);

template <class T>
int dev_upload(T** dst, const T* src, size_t n) {
  WIG_CUDA(cudaMalloc((void**)dst, n * sizeof(T)));
  if (src) WIG_CUDA(cudaMemcpy(*dst, src, n * sizeof(T), cudaMemcpyHostToDevice));
  return WIG_OK;
}

// Device allocations owned by a handle, freed together.
struct DevBuf {
  std::vector<void*> ptrs;
  template <class T> int alloc(T** p, size_t n, const T* src = nullptr) {
    int rc = dev_upload(p, src, n);
    if (rc == WIG_OK) ptrs.push_back((void*)*p);
    return rc;
  }
  void free_all() {
    for (void* p : ptrs) cudaFree(p);
    ptrs.clear();
  }
};

}  // namespace wighost
