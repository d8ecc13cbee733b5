// Dirac2D kernel entry points, compiled at run time by NVRTC for one
// propagator instance (the counterpart of GPU_Dirac2D.__init__'s SourceModule
// calls, GPU_Dirac2D.py:369-388).  The host prepends a prelude defining the
// reference's '%f' constants (mass, c, dt, dX, dY, dPx, dPy; :358-367),
// struct UserPhys { A0..A3(t, x, y) } from Potential_{0..3}_String, and the
// macros DIR_NX, DIR_NY, DIR_ROWS, DIR_RNT, DIR_RMB, DIR_C, DIR_CNT, DIR_CMB,
// DIR_SNT (DIR_RMB / DIR_CMB: resident CTAs per SM the register allocation of
// the row / column pass targets).
#pragma once
#include "wig_dirac.cuh"

__device__ __forceinline__ UserPhys user_phys(const wig::DiracArgs& a) {
  UserPhys ph;
#pragma unroll
  for (int i = 0; i < 8; ++i) ph.cf[i] = a.coef[i];
  return ph;
}

extern "C" __global__ void __launch_bounds__(DIR_RNT, DIR_RMB)
dirac_rowpass(wig::DiracArgs a, double2* psi, int mode, int parity, double t_step, double t_obs,
              double* obs_row) {
  wig::dirac_row_body<UserPhys, DIR_NX, DIR_NY, DIR_ROWS, DIR_RNT>(
      a, user_phys(a), psi, mode, parity, t_step, t_obs, obs_row);
}

extern "C" __global__ void __launch_bounds__(DIR_CNT, DIR_CMB)
dirac_colpass(wig::DiracArgs a, double2* psi) {
  wig::dirac_col_body<DIR_NX, DIR_NY, DIR_C, DIR_CNT>(a, psi);
}

extern "C" __global__ void __launch_bounds__(DIR_SNT)
dirac_final(wig::DiracArgs a, int parity, double2* scale_out) {
  wig::dirac_final_scale<DIR_SNT>(a, parity, scale_out);
}

extern "C" __global__ void __launch_bounds__(DIR_SNT)
dirac_scale(double2* psi, long n, const double2* s) {
  wig::scale_body<DIR_SNT>(psi, n, s);
}

// Absorbing-boundary factors (BaseCUDAsource_AbsorbBoundary_xy :225-283):
// j, i are the unshifted indices; w = (3 N / 100)^2.
extern "C" __global__ void dirac_setup(double* bx, double* by) {
  const int NX = DIR_NX, NY = DIR_NY;
  const double wx = pow(3. * double(NX) / 100., 2);
  const double wy = pow(3. * double(NY) / 100., 2);
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < NX; k += gridDim.x * blockDim.x) {
    const int j = (k + NX / 2) % NX;
    bx[k] = 1. - exp(-double(j * j) / wx);
    bx[NX + k] = 1. - exp(-(j - NX + 1.) * (j - NX + 1.) / wx);
  }
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < NY; k += gridDim.x * blockDim.x) {
    const int i = (k + NY / 2) % NY;
    by[k] = 1. - exp(-double(i * i) / wy);
    by[NY + k] = 1. - exp(-double((i - NY + 1) * (i - NY + 1)) / wy);
  }
}
