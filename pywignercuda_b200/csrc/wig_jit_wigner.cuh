// Wigner2D kernel entry points, compiled at run time by NVRTC for one
// propagator instance (the counterpart of the reference's SourceModule calls,
// GPU_Wigner2D_FFT.py:869-906).  The host prepends a prelude that defines
//   * the reference's kernel constants (dt, dx, dp, dtheta, dlambda, mass, hBar,
//     D_Theta, D_Lambda) as '%f'-formatted __constant__ doubles
//     (SetCUDA_Constants :833-842), visible to the user's expressions;
//   * struct UserPhys { Potential(t, x), KineticEnergy(p), f(p) } built from the
//     potential, kinetic and damping expression strings;
//   * the size / tiling macros WIG_NX, WIG_NP, WIG_XROWS, WIG_XNT,
//     WIG_KIN_STRING, WIG_PC, WIG_PNT, WIG_DAMP, WIG_RNT.
#pragma once
#ifndef WIG_PMINB
#define WIG_PMINB 3
#endif
#ifndef WIG_XMINB
#define WIG_XMINB 4
#endif
#ifndef WIG_KVN
#define WIG_KVN 0
#endif
#include "wig_wigner.cuh"

__device__ __forceinline__ UserPhys user_phys(const wig::WigArgs& a) {
  UserPhys ph;
#pragma unroll
  for (int i = 0; i < 8; ++i) ph.cf[i] = a.coef[i];
  return ph;
}

extern "C" __global__ void __launch_bounds__(WIG_XNT, WIG_XMINB)
wig_xpass(wig::WigArgs a, double2* W, int scale_mode, double* obs_row) {
  wig::xpass_body<UserPhys, WIG_NX, WIG_NP, WIG_XROWS, WIG_XNT, WIG_KIN_STRING != 0>(
      a, user_phys(a), W, scale_mode, obs_row);
}

extern "C" __global__ void __launch_bounds__(WIG_PNT, WIG_PMINB)
wig_ppass(wig::WigArgs a, double2* W, double t) {
  wig::ppass_body<UserPhys, WIG_NX, WIG_NP, WIG_PC, WIG_PNT, WIG_DAMP, WIG_KVN>(a, user_phys(a), W, t, a.partials);
}

extern "C" __global__ void __launch_bounds__(WIG_RNT)
wig_reduce(wig::WigArgs a, const double2* W) {
  wig::reduce_body<WIG_NX, WIG_NP, WIG_RNT>(a, W, a.partials);
}

extern "C" __global__ void __launch_bounds__(WIG_RNT)
wig_finalize(wig::WigArgs a, int mode, double* obs_row, double2* scale_out) {
  wig::finalize_body<WIG_RNT>(a, mode, obs_row, scale_out);
}

extern "C" __global__ void __launch_bounds__(WIG_RNT)
wig_scale(double2* W, long n, const double2* s) {
  wig::scale_body<WIG_RNT>(W, n, s);
}

extern "C" __global__ void __launch_bounds__(WIG_XNT)
wig_odm_xpass(wig::WigArgs a, const double2* W, double2* T) {
  wig::odm_xpass_body<UserPhys, WIG_NX, WIG_NP, WIG_XROWS, WIG_XNT>(a, user_phys(a), W, T);
}

extern "C" __global__ void __launch_bounds__(WIG_PNT)
wig_odm_ppass(wig::WigArgs a, double2* W, const double2* T, double coef, double sign) {
  wig::odm_ppass_body<WIG_NX, WIG_NP, WIG_PC, WIG_PNT>(a, W, T, coef, sign);
}

// Per-instance 1-D factor tables, computed on the device with the same
// expressions (and CUDA math) as the reference's kernels:
//   r_lambda  exp(-D_Lambda lambda^2)            expPLambda_source :153
//   r_theta   exp(-D_Theta theta^2 dt)           expPotential_source :117
//   mask1/2   1 - exp(-(x -+ x_max)^2/(10 dx)^2)  expPotential_source :121-123
//   sfp       sign(p) f(p)                       theta_fp_source :422-428
extern "C" __global__ void wig_setup(wig::WigArgs a, double* r_lambda, double* r_theta, double* mask1,
                                     double* mask2s, double* sfp) {
  const UserPhys ph = user_phys(a);
  const int NX = WIG_NX, NP = WIG_NP;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < NX; k += gridDim.x * blockDim.x) {
    const int jj = (k + NX / 2) % NX;
    const double lambda = dlambda * (jj - 0.5 * NX);
    r_lambda[k] = exp(-D_Lambda * lambda * lambda);
    const double x = dx * (jj - 0.5 * NX);
    const double x_max = dx * (NX - 1.) / 2.;
    mask1[k] = 1. - exp(-pow(x - x_max, 2) / pow(10. * dx, 2));
    mask2s[k] = (1. - exp(-pow(x + x_max, 2) / pow(10. * dx, 2))) * (1.0 / (double)NP);
  }
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < NP; k += gridDim.x * blockDim.x) {
    const int ii = (k + NP / 2) % NP;
    const double theta = dtheta * (ii - 0.5 * NP);
    r_theta[k] = exp(-D_Theta * theta * theta * dt);
    const double p = dp * (ii - 0.5 * NP);
    sfp[k] = (p >= 0.) ? ph.f(p) : -ph.f(p);
  }
}
