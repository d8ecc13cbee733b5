// Adjoint-form kernel entry points, compiled by NVRTC for one grid size and
// precision.  The host prepends
//   #define WIGA_NX <n_x>   #define WIGA_NP <n_p>
//   #define WIGA_PW <warps per p-pass CTA>  (a tile of 4 columns: 32- or 64-byte row segments)
//   #define WIGA_PREC 0 | 1                  (complex64 / complex128 state and transforms)
#pragma once
#include "wig_adjoint.cuh"

#ifndef WIGA_PREC
#define WIGA_PREC 0
#endif
#if WIGA_PREC == 1
typedef double2 WigaC;
#else
typedef float2 WigaC;
#endif

// x-pass: one warp per CTA (rf_spw(n_x) rows).  sgn = +1: K, -1: K^H; use_pend:
// scale the input by the pending normalisation on load.
extern "C" __global__ void __launch_bounds__(32)
wiga_xpass(wig::AArgs a, const WigaC* in, WigaC* out, double sgn, int use_pend) {
  wig::adj_xpass<WigaC, WIGA_NX, WIGA_NP>(a, in, out, sgn, use_pend);
}

// forward p-pass of step `step`: out = P(eps[step]) in, damped: C P(eps[step]) in and the
// CTA partials of its sum; U_out (may be null) receives a copy
extern "C" __global__ void __launch_bounds__(WIGA_PW * 32)
wiga_ppass(wig::AArgs a, const WigaC* in, WigaC* out, WigaC* U_out, const double* eps, long long step,
           double* part) {
  wig::adj_ppass<WigaC, WIGA_NX, WIGA_NP, WIGA_PW>(a, in, out, U_out, eps[step], part);
}

// damped forward step: s = dX dP sum U (CTA partials in order), the pending
// normalisation 1/s, and s into s_out[step] (when given).  One warp.
extern "C" __global__ void __launch_bounds__(32)
wiga_fwd_finalize(wig::AArgs a, const double* part, int n, double2* s_out, long long step) {
  double re = 0., im = 0.;
  for (int i = threadIdx.x; i < n; i += 32) { re += part[2 * i]; im += part[2 * i + 1]; }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    re += __shfl_xor_sync(0xffffffffu, re, o);
    im += __shfl_xor_sync(0xffffffffu, im, o);
  }
  if (threadIdx.x == 0) {
    const double2 s = make_double2(re * a.dx * a.dp, im * a.dx * a.dp);
    *a.pend = wig::crecip(s);
    if (s_out) s_out[step] = s;
  }
}

// W *= the pending normalisation (the end of a damped forward sweep), then pend = 1
extern "C" __global__ void __launch_bounds__(256)
wiga_scale(wig::AArgs a, WigaC* W, long long n) {
  const double2 s = *a.pend;
  const WigaC sc = wig::cmk<WigaC>(s.x, s.y);
  for (long long i = blockIdx.x * 256ll + threadIdx.x; i < n; i += (long long)gridDim.x * 256) W[i] = wig::cmul(W[i], sc);
}

extern "C" __global__ void __launch_bounds__(32)
wiga_reset_pend(wig::AArgs a) {
  if (threadIdx.x == 0) *a.pend = make_double2(1., 0.);
}

// CTA partials of sum conj(lam) U (FP64), grid-stride over the plane
extern "C" __global__ void __launch_bounds__(256)
wiga_dot(const WigaC* lam, const WigaC* U, long long n, double* part) {
  double v[2] = {0., 0.};
  for (long long i = blockIdx.x * 256ll + threadIdx.x; i < n; i += (long long)gridDim.x * 256) {
    const WigaC l = lam[i], u = U[i];
    v[0] += (double)l.x * (double)u.x + (double)l.y * (double)u.y;
    v[1] += (double)l.x * (double)u.y - (double)l.y * (double)u.x;
  }
  wig::adj_block_sum<256, 2>(v, part + 2 * blockIdx.x);
}

// The adjoint of the normalisation of step `step`: lam_U = coef[0] lam + coef[1]
// with coef[0] = 1 / conj(s), coef[1] = -conj(dX dP r / s^2), r = sum conj(lam) U.  One warp.
extern "C" __global__ void __launch_bounds__(32)
wiga_adj_coef(wig::AArgs a, const double* part, int n, const double2* s_in, long long step) {
  double re = 0., im = 0.;
  for (int i = threadIdx.x; i < n; i += 32) { re += part[2 * i]; im += part[2 * i + 1]; }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    re += __shfl_xor_sync(0xffffffffu, re, o);
    im += __shfl_xor_sync(0xffffffffu, im, o);
  }
  if (threadIdx.x == 0) {
    const double2 s = s_in[step];
    const double2 r = make_double2(re * a.dx * a.dp, im * a.dx * a.dp);
    const double2 beta = wig::cmul(r, wig::crecip(wig::cmul(s, s)));
    a.coef[0] = wig::crecip(wig::cconj(s));
    a.coef[1] = make_double2(-beta.x, beta.y);
  }
}

// adjoint p-pass of step `step`: lam <- P^H [C^H N^H] lam, gradient partials per CTA
extern "C" __global__ void __launch_bounds__(WIGA_PW * 32)
wiga_ppass_T(wig::AArgs a, WigaC* lam, const WigaC* Y, const double* eps, long long step, double* part) {
  wig::adj_ppass_T<WigaC, WIGA_NX, WIGA_NP, WIGA_PW>(a, lam, Y, eps[step], part);
}

// grad[3 step + q] = sum of the p-pass partials q in CTA order (one warp);
// q = 0: dL/d eps_step, 1: dL/dv4 share, 2: dL/dv2 share
extern "C" __global__ void __launch_bounds__(32)
wiga_grad_finalize(const double* part, int n, double* grad, long long step) {
  double s[3] = {0., 0., 0.};
  for (int i = threadIdx.x; i < n; i += 32)
#pragma unroll
    for (int q = 0; q < 3; ++q) s[q] += part[3 * i + q];
#pragma unroll
  for (int q = 0; q < 3; ++q)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s[q] += __shfl_xor_sync(0xffffffffu, s[q], o);
  if (threadIdx.x == 0)
#pragma unroll
    for (int q = 0; q < 3; ++q) grad[3 * step + q] = s[q];
}
