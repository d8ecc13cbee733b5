// Host execution of this package's CUDA device code, for checking the kernels'
// index arithmetic, tiling and synchronisation on a machine without a GPU.
// Test infrastructure only: nothing in the package includes it.
//
// One std::thread per CUDA thread; the blocks of a launch run one after another
// (the kernels checked this way never wait on another block).  __syncthreads
// is a std::barrier over the block, __syncwarp and the shuffles a barrier over
// the warp.  Block-scope `__shared__` arrays become function statics (one copy,
// seen by every thread of the running block); `extern __shared__` arrays are
// rewritten by the test harness to point into emu_smem.  Math functions are
// the host C library's.  Blocks running one after another, a persistent
// kernel's first block drains its work list and the others draw only the
// overflowing tickets.
#pragma once
#include <math.h>

#include <atomic>
#include <cmath>
#include <cstdint>
#include <barrier>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <memory>
#include <new>
#include <thread>
#include <vector>

struct double2 { double x, y; };
struct float2 { float x, y; };
struct int2 { int x, y; };
inline double2 make_double2(double a, double b) { return {a, b}; }
inline float2 make_float2(float a, float b) { return {a, b}; }
inline int2 make_int2(int a, int b) { return {a, b}; }

struct emu_dim3 { unsigned x = 0, y = 1, z = 1; };
inline thread_local emu_dim3 threadIdx, blockIdx;
inline emu_dim3 blockDim, gridDim;

#define __device__
#define __host__
#define __global__
#define __forceinline__ inline
#define __restrict__
#define __launch_bounds__(...)
#define __shared__ static
#define __grid_constant__
#define __align__(n) __attribute__((aligned(n)))

inline unsigned char* emu_smem = nullptr;   // the running launch's dynamic shared memory
struct emu_aligned_delete {
  void operator()(unsigned char* p) const { ::operator delete[](p, std::align_val_t(256)); }
};

inline std::barrier<>* emu_block_barrier = nullptr;
inline std::vector<std::unique_ptr<std::barrier<>>> emu_warp_barriers;
inline double emu_shfl[1024];

inline void __syncthreads() { emu_block_barrier->arrive_and_wait(); }
inline void __syncwarp(unsigned = 0xffffffffu) { emu_warp_barriers[threadIdx.x / 32]->arrive_and_wait(); }

// every lane of the warp takes part (the kernels shuffle with full masks only)
inline double __shfl_xor_sync(unsigned, double v, int lane_mask) {
  const unsigned t = threadIdx.x;
  std::barrier<>& wb = *emu_warp_barriers[t / 32];
  emu_shfl[t] = v;
  wb.arrive_and_wait();
  const double r = emu_shfl[(t & ~31u) | ((t & 31u) ^ (unsigned)lane_mask)];
  wb.arrive_and_wait();
  return r;
}

template <class T> inline T __ldg(const T* p) { return *p; }
template <class T> inline T __ldcg(const T* p) { return *p; }

inline unsigned atomicAdd(unsigned* p, unsigned v) { return std::atomic_ref<unsigned>(*p).fetch_add(v); }
inline int atomicExch(int* p, int v) { return std::atomic_ref<int>(*p).exchange(v); }
inline void __threadfence() { std::atomic_thread_fence(std::memory_order_seq_cst); }

// sin / cos of pi x, evaluated in double and rounded once
inline void sincospif(float x, float* s, float* c) {
  const double a = 3.141592653589793238462643383279502884 * (double)x;
  *s = (float)::sin(a);
  *c = (float)::cos(a);
}

// sin / cos of pi x in double, from extended precision
inline void sincospi(double x, double* s, double* c) {
  const long double a = 3.141592653589793238462643383279502884L * (long double)x;
  *s = (double)::sinl(a);
  *c = (double)::cosl(a);
}

// bit casts, and the double -> float conversion rounding toward zero
inline long long __double_as_longlong(double v) {
  long long b;
  std::memcpy(&b, &v, sizeof b);
  return b;
}
inline double __longlong_as_double(long long b) {
  double v;
  std::memcpy(&v, &b, sizeof v);
  return v;
}
inline float __double2float_rz(double v) {
  float f = (float)v;
  if (std::isfinite(f) && std::fabs((double)f) > std::fabs(v)) f = std::nextafterf(f, 0.f);
  return f;
}

// (grid_x, grid_y) x block threads; a block's threads run concurrently, blocks in turn.
// smem: bytes of dynamic shared memory (0: a 4 MiB buffer, for kernels with none).
inline void emu_launch2d(unsigned grid_x, unsigned grid_y, unsigned block, const std::function<void()>& body,
                         size_t smem = 0) {
  if (block == 0 || block > 1024 || (block % 32) != 0) {
    std::fprintf(stderr, "emu_launch: block of %u threads\n", block);
    std::exit(3);
  }
  const size_t bytes = smem ? smem : ((size_t)1 << 22);
  std::unique_ptr<unsigned char[], emu_aligned_delete> buf(new (std::align_val_t(256)) unsigned char[bytes]);
  gridDim = {grid_x, grid_y, 1};
  blockDim = {block, 1, 1};
  for (unsigned by = 0; by < grid_y; ++by)
    for (unsigned bx = 0; bx < grid_x; ++bx) {
      std::memset(buf.get(), 0xff, bytes);
      emu_smem = buf.get();
      std::barrier<> bar((std::ptrdiff_t)block);
      emu_block_barrier = &bar;
      emu_warp_barriers.clear();
      for (unsigned w = 0; w < block / 32; ++w) emu_warp_barriers.emplace_back(new std::barrier<>(32));
      std::vector<std::thread> threads;
      threads.reserve(block);
      for (unsigned t = 0; t < block; ++t)
        threads.emplace_back([&body, t, bx, by] {
          threadIdx = {t, 0, 0};
          blockIdx = {bx, by, 0};
          body();
        });
      for (auto& th : threads) th.join();
    }
}

inline void emu_launch(unsigned grid, unsigned block, const std::function<void()>& body, size_t smem = 0) {
  emu_launch2d(grid, 1, block, body, smem);
}

// WIG_BOUNDS: an index check of the device code failed
inline void wig_bounds_fail(const char* what, long long i, long long n) {
  std::fprintf(stderr, "WIG_BOUNDS: %s index %lld outside [0, %lld)\n", what, i, n);
  std::abort();
}
