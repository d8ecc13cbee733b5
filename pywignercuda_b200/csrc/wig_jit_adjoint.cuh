// Adjoint-form kernel entry points, compiled by NVRTC for one grid size.  The
// host prepends
//   #define WIGA_NX <n_x>   #define WIGA_NP <n_p>
//   #define WIGA_PW <warps per p-pass CTA>  (a tile of 4 columns: 32-byte row segments)
#pragma once
#include "wig_adjoint.cuh"

// x-pass: one warp per CTA (rf_spw(n_x) rows).  sgn = +1: K, -1: K^H.
extern "C" __global__ void __launch_bounds__(32)
wiga_xpass(wig::AArgs a, const float2* in, float2* out, float sgn) {
  wig::adj_xpass<WIGA_NX, WIGA_NP>(a, in, out, sgn);
}

// forward p-pass of step `step`: out = P(eps[step]) in
extern "C" __global__ void __launch_bounds__(WIGA_PW * 32)
wiga_ppass(wig::AArgs a, const float2* in, float2* out, const double* eps, long long step) {
  wig::adj_ppass<WIGA_NX, WIGA_NP, WIGA_PW>(a, in, out, eps[step]);
}

// adjoint p-pass of step `step`: lam <- P(eps[step])^H lam, gradient partials per CTA
extern "C" __global__ void __launch_bounds__(WIGA_PW * 32)
wiga_ppass_T(wig::AArgs a, float2* lam, const float2* Y, const double* eps, long long step, double* partials) {
  wig::adj_ppass_T<WIGA_NX, WIGA_NP, WIGA_PW>(a, lam, Y, eps[step], partials);
}

// grad[step] = sum of the p-pass partials in CTA order (one warp)
extern "C" __global__ void __launch_bounds__(32)
wiga_grad_finalize(const double* partials, int n, double* grad, long long step) {
  double s = 0.;
  for (int i = threadIdx.x; i < n; i += 32) s += partials[i];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (threadIdx.x == 0) grad[step] = s;
}
