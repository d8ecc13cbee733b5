// Batched FP32 Wigner2D kernel entry points, compiled by NVRTC for one batch
// (its set of grid-size classes and tile shape).  The host prepends
//   #define WIGB_WARPS <warps per CTA>   (the autotuned tile shape)
//   #define WIGB_CASES(F) F(128) F(256) ...   (the size classes present)
//   #define WIGB_PREC 0 | 1                      (FP32 / mixed precision, wig_batch.cuh)
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
template <int N> __device__ WIGB_CASE_INLINE void wigb_x_case(const wig::BArgs& A, int inst, const wig::BInst& I, int row0) {
  wig::batch_x_item<N>(A, inst, I, row0);
}
template <int N> __device__ WIGB_CASE_INLINE void wigb_p_case(const wig::BArgs& A, int inst, const wig::BInst& I, int col0,
                                                          int item, int sample) {
  wig::batch_p_item<N>(A, inst, I, col0, item, sample);
}
#define WIGB_X_CASE(N) case N: wigb_x_case<N>(A, it.x, sI, it.y); break;
#define WIGB_P_CASE(N) case N: wigb_p_case<N>(A, it.x, sI, it.y, item, sample); break;
#define WIGB_R_CASE(N) case N: wig::batch_reduce_item<N>(A, it.x, sI, it.y, item, mode, sample); break;
#define WIGB_S_CASE(N) case N: wig::batch_scale_item<N>(A, it.x, sI, it.y); break;

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
