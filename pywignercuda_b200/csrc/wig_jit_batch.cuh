// Batched FP32 Wigner2D kernel entry points, compiled by NVRTC for one batch
// (its set of grid-size classes and tile shape).  The host prepends
//   #define WIGB_WARPS <warps per CTA>   (the autotuned tile shape)
//   #define WIGB_CASES(F) F(128) F(256) ...   (the size classes present)
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

#define WIGB_X_CASE(N) case N: wig::batch_x_item<N>(A, it.x, sI, it.y); break;
#define WIGB_P_CASE(N) case N: wig::batch_p_item<N>(A, it.x, sI, it.y, item, sample); break;
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
