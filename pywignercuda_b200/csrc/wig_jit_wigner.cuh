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
#ifndef WIG_STRANG
#define WIG_STRANG 0
#endif
#ifndef WIG_RF
#define WIG_RF 0
#endif
#include "wig_wigner.cuh"
#include "wig_wigner_rf.cuh"

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

#if WIG_RF
// The Lie step's passes on the register-resident FFT (wig_wigner_rf.cuh): WIG_RFXW
// warps per x-pass CTA (rf_spw(n_x) rows each), WIG_RFPW warps per p-pass CTA
// (rf_spw(n_p) columns each); the host picks them instead of wig_xpass /
// wig_ppass for Lie plans without ODM damping on grids of 64 to 1024 points.
extern "C" __global__ void __launch_bounds__(WIG_RFXW * 32, WIG_RFXMB)
wig_xpass_rf(wig::WigArgs a, double2* W, int scale_mode, double* obs_row) {
  wig::xpass_rf_body<UserPhys, WIG_NX, WIG_NP, WIG_RFXW, WIG_KIN_STRING != 0>(a, user_phys(a), W, scale_mode,
                                                                              obs_row);
}

// map: the tensor map of W for the tile's 2-D tensor copies (used when WIG_TMA is defined)
extern "C" __global__ void __launch_bounds__(WIG_RFPW * 32, WIG_RFPMB)
wig_ppass_rf(wig::WigArgs a, double2* W, double t, const __grid_constant__ wig::TensorMap map) {
  wig::ppass_rf_body<UserPhys, WIG_NX, WIG_NP, WIG_RFPW, WIG_DAMP, WIG_KVN>(a, user_phys(a), W, t, a.partials, &map);
}
#endif

#if WIG_STRANG
// Strang-split step of GPU_Wigner2D_GPitaevskii (:1897-1975): first half p-pass
// (consumes the previous partials, normalises on load, records the sample),
// then -- after the kinetic x-pass -- the final half p-pass with the damping
// and the partial sums.  gp_phase: the Gross-Pitaevskii phase array or null.
extern "C" __global__ void __launch_bounds__(WIG_PNT, WIG_PMINB)
wig_ppass_half(wig::WigArgs a, double2* W, double t, int scale_mode, double* obs_row, const double* gp_phase) {
  wig::ppass_body<UserPhys, WIG_NX, WIG_NP, WIG_PC, WIG_PNT, 0, 0, 1, 0>(a, user_phys(a), W, t, a.partials,
                                                                        scale_mode, obs_row, gp_phase);
}

extern "C" __global__ void __launch_bounds__(WIG_PNT, WIG_PMINB)
wig_ppass_half_final(wig::WigArgs a, double2* W, double t, const double* gp_phase) {
  wig::ppass_body<UserPhys, WIG_NX, WIG_NP, WIG_PC, WIG_PNT, WIG_DAMP, 0, 1, 1>(a, user_phys(a), W, t, a.partials,
                                                                                0, nullptr, gp_phase);
}

#define WIG_GP_RCH 16
#define WIG_GP_CNT (WIG_NX < 256 ? WIG_NX : 256)
extern "C" __global__ void __launch_bounds__(WIG_GP_CNT)
wig_gp_colsum(const double2* W, double2* chunks) {
  wig::colsum_body<WIG_NX, WIG_NP, WIG_GP_RCH, WIG_GP_CNT>(W, chunks);
}

extern "C" __global__ void __launch_bounds__(256)
wig_gp_marginal(wig::WigArgs a, const double2* chunks, int n_chunks, int scale_mode, double* P, double* psq) {
  wig::gp_marginal_body<WIG_NX, 256>(a, chunks, n_chunks, scale_mode, P, psq);
}

extern "C" __global__ void __launch_bounds__(WIG_XNT)
wig_gp_phase(wig::WigArgs a, const double* P, double* phase_out) {
  wig::gp_phase_body<WIG_NX, WIG_NP, WIG_XROWS, WIG_XNT>(a, P, phase_out);
}

// Bloch (imaginary-time) step pieces, GPU_Wigner2D_GPitaevskii_Bloch (:2064-2545)
extern "C" __global__ void __launch_bounds__(WIG_PNT, WIG_PMINB)
wig_bloch_ppass(wig::WigArgs a, double2* W, double t, double dtb, const double* gexp) {
  wig::bloch_ppass_body<UserPhys, WIG_NX, WIG_NP, WIG_PC, WIG_PNT>(a, user_phys(a), W, t, dtb, gexp);
}

extern "C" __global__ void __launch_bounds__(WIG_XNT, WIG_XMINB)
wig_bloch_xpass(wig::WigArgs a, double2* W, double dtb) {
  wig::bloch_xpass_body<UserPhys, WIG_NX, WIG_NP, WIG_XROWS, WIG_XNT>(a, user_phys(a), W, dtb);
}

extern "C" __global__ void __launch_bounds__(WIG_XNT)
wig_gp_bloch(wig::WigArgs a, const double* P, double dtb, double* out) {
  wig::gp_bloch_body<WIG_NX, WIG_NP, WIG_XROWS, WIG_XNT>(a, P, dtb, out);
}

extern "C" __global__ void __launch_bounds__(WIG_RNT)
wig_bloch_reduce(wig::WigArgs a, const double2* W, const double2* W0, double* partials) {
  wig::bloch_reduce_body<UserPhys, WIG_NX, WIG_NP, WIG_RNT>(a, user_phys(a), W, W0, partials);
}

extern "C" __global__ void __launch_bounds__(256)
wig_rowsum(const double2* W, double2* out) {
  wig::rowsum_body<WIG_NX, 256>(W, out);
}

extern "C" __global__ void __launch_bounds__(WIG_RNT)
wig_bloch_axpy(double2* W, const double2* W0, long n, double2 c, double2 s) {
  wig::bloch_axpy_body<WIG_RNT>(W, W0, n, c, s);
}
#endif

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
//   r_theta_half exp(-0.5 D_Theta theta^2 dt)    (Strang half step)
extern "C" __global__ void wig_setup(wig::WigArgs a, double* r_lambda, double* r_theta, double* mask1,
                                     double* mask2s, double* sfp, double* r_theta_half) {
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
    r_theta_half[k] = exp(-0.5 * D_Theta * theta * theta * dt);   // GPU_Wigner2D_GPitaevskii :66
    const double p = dp * (ii - 0.5 * NP);
    sfp[k] = (p >= 0.) ? ph.f(p) : -ph.f(p);
  }
}
