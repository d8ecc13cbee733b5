// Batched FP32 Wigner2D kernel entry points, compiled by NVRTC for one batch
// (its set of grid-size classes and tile shape).  The host prepends
//   #define WIGB_WARPS <warps per CTA>   (the autotuned tile shape)
//   #define WIGB_CASES(F) F(128) F(256) ...   (the size classes present)
//   #define WIGB_PREC 0 | 1                      (FP32 / mixed precision, wig_batch.cuh)
//   #define WIGB_XSTAGE 0 | 1                    (x-pass rows staged in shared memory)
// Each kernel is persistent over its work list: the x- and p-pass draw items
// from a ticket counter, the one-off reduce / scale kernels take items
// b, b + gridDim.x, ...
#pragma once
#include "wig_batch.cuh"

#ifndef WIGB_XMINB
#define WIGB_XMINB 1
#endif
#ifndef WIGB_PMINB
#define WIGB_PMINB 1
#endif

// WIGB_NOINLINE 1: each size class's pass body is its own (non-inlined)
// function, so registers are allocated per class rather than over the union of
// every class's code (at the cost of a call and a stack frame per item).
#ifndef WIGB_NOINLINE
#define WIGB_NOINLINE 0
#endif
#if WIGB_NOINLINE
#define WIGB_CASE_INLINE __noinline__
#else
#define WIGB_CASE_INLINE __forceinline__
#endif
template <int N> __device__ WIGB_CASE_INLINE void wigb_p_case(const wig::BArgs& A, int inst, const wig::BInst& I, int col0,
                                                          int item, int sample) {
  wig::batch_p_item<N>(A, inst, I, col0, item, sample);
}
#define WIGB_P_CASE(N) case N: wigb_p_case<N>(A, it.x, sI, it.y, item, sample); break;
#define WIGB_R_CASE(N) case N: wig::batch_reduce_item<N>(A, it.x, sI, it.y, item, mode, sample); break;
#define WIGB_S_CASE(N) case N: wig::batch_scale_item<N>(A, it.x, sI, it.y); break;

// ---------------------------------------------------------------- x-pass row staging
// The x-pass is persistent over its work list, and each item's rows are one
// contiguous block of W: while a CTA transforms an item, the next item's rows
// are already on their way into a staging buffer in shared memory.  With
// WIGB_BULK (the library's GPU build) the block arrives by a bulk asynchronous
// copy (cp.async.bulk, completing on an mbarrier; no multicast); the wait is
// bounded and, when it gives up, records 1 in A.status (the host reports
// WIG_ERR_TIMEOUT).  Without it (host execution of this code) thread 0 copies
// the block, ordered by the CTA's barriers.
#define WIGB_XEXCH_F(N) m = m > wig::bx_exch(N, WIGB_WARPS, WIGB_PREC) ? m : wig::bx_exch(N, WIGB_WARPS, WIGB_PREC);
#define WIGB_XSTAGE_F(N) m = m > wig::bx_stage(N, WIGB_WARPS) ? m : wig::bx_stage(N, WIGB_WARPS);
__host__ __device__ constexpr int wigb_xexch_max() {
  int m = 0;
  WIGB_CASES(WIGB_XEXCH_F)
  return m;
}
__host__ __device__ constexpr int wigb_xstage_max() {
  int m = 0;
  WIGB_CASES(WIGB_XSTAGE_F)
  return m;
}

// Polls of a staging wait before it gives up.
#ifndef WIGB_WAIT_POLLS
#define WIGB_WAIT_POLLS (1L << 24)
#endif

#ifdef WIGB_BULK
__device__ __forceinline__ unsigned wigb_smem(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void wigb_stage_init(unsigned long long* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(wigb_smem(bar)) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// WIGB_TEST_STALL (failure-detection tests only): the copy is announced to the
// mbarrier but never issued, so every wait runs out -- nothing is in flight
// when the kernel gives up and returns.
__device__ __forceinline__ void wigb_stage_copy(float* dst, const float* src, unsigned bytes, unsigned long long* bar) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(wigb_smem(bar)), "r"(bytes) : "memory");
#ifndef WIGB_TEST_STALL
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   wigb_smem(dst)),
               "l"(src), "r"(bytes), "r"(wigb_smem(bar))
               : "memory");
#endif
}
// Bounded wait for the staged rows: after WIGB_WAIT_POLLS polls it records 1 in
// the status word (the host reports WIG_ERR_TIMEOUT) and sets the CTA's `stalled`
// flag, after which the CTA issues no further copies and its later waits return
// at once (the run is already failed; the items are still drawn, so the work list
// ends in its usual state).
__device__ __forceinline__ void wigb_stage_wait(unsigned long long* bar, unsigned phase, unsigned* status,
                                                volatile int* stalled) {
  if (*stalled) return;
  unsigned done = 0;
#pragma unroll 1
  for (long it = 0; it < WIGB_WAIT_POLLS && !done; ++it)
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(wigb_smem(bar)), "r"(phase)
        : "memory");
  if (!done) {
    *stalled = 1;
    if (threadIdx.x == 0) atomicExch(status, 1u);
  }
}
#else
__device__ __forceinline__ void wigb_stage_init(unsigned long long*) {}
__device__ __forceinline__ void wigb_stage_copy(float* dst, const float* src, unsigned bytes, unsigned long long*) {
  memcpy(dst, src, bytes);
}
__device__ __forceinline__ void wigb_stage_wait(unsigned long long*, unsigned, unsigned*, volatile int*) {}
#endif

// WIGB_XSTAGE 1: the staged x-pass above; 0: each lane loads its rows from
// global memory directly (no staging buffer: less shared memory a CTA, and
// the loads are in flight only while the CTA waits on them).
#ifndef WIGB_XSTAGE
#define WIGB_XSTAGE 1
#endif

#if WIGB_XSTAGE
#define WIGB_X_CASE(N) case N: wig::batch_x_item_t<wig::XC, N>(A, sIn[buf], sI[buf], sRow[buf], stage, after); break;

// Shared memory: the exchange regions (wigb_xexch_max() float2), then the
// staging buffer (wigb_xstage_max() floats).
extern "C" __global__ void __launch_bounds__(WIGB_NT, WIGB_XMINB)
wigb_xpass(wig::BArgs A, int n_items) {
  extern __shared__ float2 smb[];
  float* stage = reinterpret_cast<float*>(smb + wigb_xexch_max());
  __shared__ wig::BInst sI[2];
  __shared__ int sIn[2], sRow[2];
  __shared__ __align__(8) unsigned long long bar;
  __shared__ volatile int stalled;
  int item = wig::next_item(&A.tickets[0], n_items);
  int buf = 0;
  unsigned phase = 0;
  // the first item's rows
  if (threadIdx.x == 0) {
    stalled = 0;
    wigb_stage_init(&bar);
    if (item < n_items) {
      const int2 it = A.xitems[item];
      sI[0] = A.inst[it.x];
      sIn[0] = it.x;
      sRow[0] = it.y;
      wigb_stage_copy(stage, A.W + sI[0].off + (size_t)it.y * sI[0].n_x,
                      (unsigned)(wig::bx_stage(sI[0].n_x, WIGB_WARPS) * sizeof(float)), &bar);
    }
  }
  __syncthreads();
  while (item < n_items) {
    wigb_stage_wait(&bar, phase, A.status, &stalled);
    int next = n_items;
    // every lane holds its rows: draw the next item and start its rows' copy
    auto after = [&]() {
      __syncthreads();
      next = wig::next_item(&A.tickets[0], n_items);
      if (threadIdx.x == 0 && next < n_items) {
        const int2 it = A.xitems[next];
        sI[buf ^ 1] = A.inst[it.x];
        sIn[buf ^ 1] = it.x;
        sRow[buf ^ 1] = it.y;
        // after a wait gave up, the barrier's phase never completes: no further arrival
        // (it would arrive on a phase with no pending arrivals) and no further copy
        if (!stalled)
          wigb_stage_copy(stage, A.W + sI[buf ^ 1].off + (size_t)it.y * sI[buf ^ 1].n_x,
                          (unsigned)(wig::bx_stage(sI[buf ^ 1].n_x, WIGB_WARPS) * sizeof(float)), &bar);
      }
    };
    switch (sI[buf].n_x) {
      WIGB_CASES(WIGB_X_CASE)
      default: after(); break;
    }
    __syncthreads();   // the item's exchange reads are done; sI[buf ^ 1] is visible
    item = next;
    buf ^= 1;
    phase ^= 1u;
  }
}
#else
#define WIGB_X_CASE(N)                                                                              \
  case N:                                                                                           \
    wig::batch_x_item_t<wig::XC, N>(A, it.x, sI, it.y, A.W + sI.off + (size_t)it.y * N, [] {}); \
    break;

// Shared memory: the exchange regions (wigb_xexch_max() float2).
extern "C" __global__ void __launch_bounds__(WIGB_NT, WIGB_XMINB)
wigb_xpass(wig::BArgs A, int n_items) {
  __shared__ wig::BInst sI;
  for (int item = wig::next_item(&A.tickets[0], n_items); item < n_items;
       item = wig::next_item(&A.tickets[0], n_items)) {
    const int2 it = A.xitems[item];
    if (threadIdx.x == 0) sI = A.inst[it.x];
    __syncthreads();
    switch (sI.n_x) { WIGB_CASES(WIGB_X_CASE) default: break; }
    __syncthreads();
  }
}
#endif

extern "C" __global__ void __launch_bounds__(WIGB_NT, WIGB_PMINB)
wigb_ppass(wig::BArgs A, int n_items, int sample) {
  __shared__ wig::BInst sI;
  for (int item = wig::next_item(&A.tickets[1], n_items); item < n_items;
       item = wig::next_item(&A.tickets[1], n_items)) {
    const int2 it = A.pitems[item];
    if (threadIdx.x == 0) sI = A.inst[it.x];
    __syncthreads();
    switch (sI.n_p) { WIGB_CASES(WIGB_P_CASE) default: break; }
    __syncthreads();
  }
}

extern "C" __global__ void __launch_bounds__(WIGB_NT)
wigb_reduce(wig::BArgs A, int n_items, int mode, int sample) {
  __shared__ wig::BInst sI;
  for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
    const int2 it = A.pitems[item];
    if (threadIdx.x == 0) sI = A.inst[it.x];
    __syncthreads();
    switch (sI.n_p) { WIGB_CASES(WIGB_R_CASE) default: break; }
    __syncthreads();
  }
}

extern "C" __global__ void __launch_bounds__(WIGB_NT)
wigb_scale(wig::BArgs A, int n_items) {
  __shared__ wig::BInst sI;
  for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
    const int2 it = A.pitems[item];
    if (threadIdx.x == 0) sI = A.inst[it.x];
    __syncthreads();
    switch (sI.n_p) { WIGB_CASES(WIGB_S_CASE) default: break; }
    __syncthreads();
  }
}
