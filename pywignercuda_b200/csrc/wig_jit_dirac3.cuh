// Dirac3D kernel entry points, compiled at run time by NVRTC for one propagator
// instance (the counterpart of GPU_Dirac3D.__init__'s SourceModule calls,
// GPU_Dirac3D.py:706-757).  The host prepends a prelude defining the
// reference's '%f' constants, struct UserPhys { A0..A3(t, x, y, z) } from
// Potential_{0..3}_String, and the macros D3_NX, D3_NY, D3_NZ, D3_ROWS,
// D3_XNT, D3_YC, D3_YNT, D3_ZC, D3_ZNT, D3_SNT.
#pragma once
#include "wig_dirac3.cuh"

__device__ __forceinline__ UserPhys user_phys(const wig::Dirac3Args& a) {
  UserPhys ph;
#pragma unroll
  for (int i = 0; i < 8; ++i) ph.cf[i] = a.coef[i];
  return ph;
}

// D3_XMB / D3_YMB / D3_ZMB: resident CTAs per SM the register allocation targets;
// D3_XR / D3_YR / D3_ZR: largest Stockham radix of each pass's transforms
extern "C" __global__ void __launch_bounds__(D3_XNT, D3_XMB)
d3_xpass(wig::Dirac3Args a, double2* psi, int mode, int parity, int normalise, double t_A, double t_obs,
         long long prev_tindex, double* obs_prev) {
  wig::d3_xpass_body<UserPhys, D3_NX, D3_NY, D3_NZ, D3_ROWS, D3_XNT, D3_XR>(a, user_phys(a), psi, mode, parity, normalise,
                                                                    t_A, t_obs, prev_tindex, obs_prev);
}

extern "C" __global__ void __launch_bounds__(D3_YNT, D3_YMB) d3_ypass_fwd(wig::Dirac3Args a, double2* psi) {
  wig::d3_ypass_body<D3_NX, D3_NY, D3_NZ, D3_YC, D3_YNT, false, D3_YR>(a, psi);
}

extern "C" __global__ void __launch_bounds__(D3_YNT, D3_YMB) d3_ypass_inv(wig::Dirac3Args a, double2* psi) {
  wig::d3_ypass_body<D3_NX, D3_NY, D3_NZ, D3_YC, D3_YNT, true, D3_YR>(a, psi);
}

extern "C" __global__ void __launch_bounds__(D3_ZNT, D3_ZMB) d3_zpass(wig::Dirac3Args a, double2* psi) {
  wig::d3_zpass_body<D3_NX, D3_NY, D3_NZ, D3_ZC, D3_ZNT, D3_ZR>(a, psi);
}

extern "C" __global__ void __launch_bounds__(D3_SNT) d3_norm(wig::Dirac3Args a, const double2* psi, long n) {
  wig::d3_norm_body<D3_SNT>(a, psi, n);
}

extern "C" __global__ void __launch_bounds__(D3_SNT) d3_norm_fin(wig::Dirac3Args a, int n_cta) {
  wig::d3_norm_final<D3_SNT>(a, n_cta);
}
