// Host-side set-up of the batched form (wigb_create): the register-FFT twiddle
// tables and each instance's constants and factor tables.  Included by the
// library (wig_capi.cu) and by the host execution of the device code
// (tests/emu/batch_emu.cpp), so both build identical tables.
#pragma once
#include <math.h>

#include <map>
#include <vector>

#include "wig_batch.cuh"

namespace wighost {

// exp(-2 pi i m / n) as a float pair: among the pairs within 2 ulp of the
// extended-precision value, the one with |w|^2 closest to 1 (ties: the closest
// in angle).  A forward twiddle and its conjugate in the inverse transform then
// leave the spectral component's magnitude unbiased.
inline float2 twiddle_f(int n, long long m) {
  const long double pi = 3.141592653589793238462643383279502884L;
  const long double a = 2.0L * pi * (long double)(m % n) / (long double)n;
  const long double c = cosl(a), s = -sinl(a);
  const float c0 = (float)c, s0 = (float)s;
  float bc = c0, bs = s0;
  long double best = 1e30L;
  for (int i = -2; i <= 2; ++i)
    for (int j = -2; j <= 2; ++j) {
      float cc = c0, ss = s0;
      for (int k = 0; k < (i < 0 ? -i : i); ++k) cc = nextafterf(cc, i > 0 ? 2.f : -2.f);
      for (int k = 0; k < (j < 0 ? -j : j); ++k) ss = nextafterf(ss, j > 0 ? 2.f : -2.f);
      const long double d = fabsl((long double)cc * cc + (long double)ss * ss - 1.0L);
      const long double key = d + 1e-3L * (fabsl((long double)cc - c) + fabsl((long double)ss - s));
      if (key < best) { best = key; bc = cc; bs = ss; }
    }
  return make_float2(bc, bs);
}

// exp(-2 pi i m / n) rounded to double from extended precision
inline double2 twiddle_d(int n, long long m) {
  const long double pi = 3.141592653589793238462643383279502884L;
  const long double a = 2.0L * pi * (long double)(m % n) / (long double)n;
  return make_double2((double)cosl(a), (double)(-sinl(a)));
}

// Register-FFT tables of length n (wig_rfft.cuh): forward tf[a G + g] = W^{g a},
// then inverse ti[(i G + b) G + t] = W^{b (t Q + i)}; 2 n entries.
template <class C, class F>
void rf_twiddles_t(int n, std::vector<C>* tw, F w) {
  const int E = wig::rf_e(n), G = wig::rf_g(n), Q = E / G;
  for (int a = 0; a < E; ++a)
    for (int g = 0; g < G; ++g) tw->push_back(w(n, (long long)g * a));
  for (int i = 0; i < Q; ++i)
    for (int b = 0; b < G; ++b)
      for (int t = 0; t < G; ++t) tw->push_back(w(n, (long long)b * (t * Q + i)));
}
inline void rf_twiddles(int n, std::vector<float2>* tw) { rf_twiddles_t(n, tw, twiddle_f); }
inline void rf_twiddles64(int n, std::vector<double2>* tw) { rf_twiddles_t(n, tw, twiddle_d); }

// One batched instance: constants of BInst (b.off, b.tw_*, work-list fields
// are set by the caller) and its factor tables, appended to ft (FP32) and fd
// (FP64; offsets kept even so the double2 sub-table is 16-byte aligned).
//   ft at ft_x: [r_lambda / n_x][mask1 mask2 / n_p][(cos, -sin) of the row-pair kinetic ratio]
//   ft at ft_p: [r_theta][sign(p) f(p)][theta / n_p]
//   fd at fd_x: [r_lambda / n_x][mask1 mask2 / n_p][(cos, -sin) of the row-pair kinetic ratio]
//   fd at fd_p: [r_theta][sign(p) f(p)][theta / n_p]
// (expPLambda_source :153, expPotential_source :117-123, theta_fp_source
// :422-428 of GPU_Wigner2D_FFT.py; every entry formed in FP64.)
// D: any struct with the fields of wigb_instance.
template <class D>
void batch_instance_setup(const D& d, wig::BInst& b, std::vector<float>* ft, std::vector<double>* fd) {
  b.n_x = d.n_x;
  b.n_p = d.n_p;
  b.damp = d.gamma != 0. ? 1 : 0;
  b.ff = d.damping_f;
  b.dt = d.dt;
  b.hbar = d.hbar;
  b.mass = d.mass;
  b.dx = 2. * d.x_amplitude / d.n_x;
  b.dp = 2. * d.p_amplitude / d.n_p;
  b.dtheta = 2. * M_PI / (2. * d.p_amplitude);
  b.dlambda = 2. * M_PI / (2. * d.x_amplitude);
  b.D_theta = d.d_theta;
  b.D_lambda = d.d_lambda;
  b.f_eps = d.f_eps;
  b.v4 = d.v4; b.v2 = d.v2; b.v1 = d.v1; b.v0 = d.v0;
  // CaldeiraDissipatorOrder3 (GPU_Wigner2D_FFT.py:1145-1157) in Horner form, imaginary parts
  const double g = d.dt * d.gamma, c1 = 2. / 3. * g, c2 = g, c3 = 2. * g;
  b.cl_k1 = (c1 + c2) != 0. ? c1 * c2 / (c1 + c2) : 0.;
  b.cl_k12 = c1 + c2;
  b.cl_c3 = c3;
  const int nx = d.n_x, np = d.n_p;
  std::vector<double> rl(nx), mm(nx), gc(nx), gs(nx), rt(np), sf(np), th(np);
  for (int k = 0; k < nx; ++k) {
    const double lam = b.dlambda * (((k + nx / 2) % nx) - 0.5 * nx);
    rl[k] = exp(-b.D_lambda * lam * lam) / (double)nx;
  }
  const double x_max = b.dx * (nx - 1.) / 2.;
  for (int k = 0; k < nx; ++k) {
    const double x = b.dx * (((k + nx / 2) % nx) - 0.5 * nx);
    const double w2 = (10. * b.dx) * (10. * b.dx);
    const double m1 = 1. - exp(-(x - x_max) * (x - x_max) / w2), m2 = 1. - exp(-(x + x_max) * (x + x_max) / w2);
    mm[k] = m1 * m2 / (double)np;
  }
  // exp(-i dt dp lambda / m) per x-frequency: the kinetic factor of row p + dp over that of
  // row p (the x-pass carries rows 2r and 2r + 1 together), as (cos, -sin) of the turn
  for (int k = 0; k < nx; ++k) {
    const int lj = k < nx / 2 ? k : k - nx;
    double t = b.dt * b.dp * b.dlambda * (double)lj / (b.mass * 2. * M_PI);
    t -= rint(t);
    gc[k] = cos(2. * M_PI * t);
    gs[k] = -sin(2. * M_PI * t);
  }
  for (int k = 0; k < np; ++k) {
    const double thk = b.dtheta * (((k + np / 2) % np) - 0.5 * np);
    rt[k] = exp(-b.D_theta * thk * thk * b.dt);
    th[k] = thk / (double)np;
    const double p = b.dp * (((k + np / 2) % np) - 0.5 * np);
    const double f = b.ff == 0 ? fabs(p) : p * p / sqrt(p * p + b.f_eps);
    sf[k] = p >= 0. ? f : -f;
  }
  b.ft_x = (int)ft->size();
  for (double v : rl) ft->push_back((float)v);
  for (double v : mm) ft->push_back((float)v);
  for (int k = 0; k < nx; ++k) { ft->push_back((float)gc[k]); ft->push_back((float)gs[k]); }
  b.ft_p = (int)ft->size();
  for (double v : rt) ft->push_back((float)v);
  for (double v : sf) ft->push_back((float)v);
  for (double v : th) ft->push_back((float)v);
  if (fd->size() & 1) fd->push_back(0.);
  b.fd_x = (int)fd->size();
  for (double v : rl) fd->push_back(v);
  for (double v : mm) fd->push_back(v);
  for (int k = 0; k < nx; ++k) { fd->push_back(gc[k]); fd->push_back(gs[k]); }
  b.fd_p = (int)fd->size();
  for (double v : rt) fd->push_back(v);
  for (double v : sf) fd->push_back(v);
  for (double v : th) fd->push_back(v);
}

// Twiddle tables of every size class (float and double, same offsets).
inline void batch_twiddles(const std::vector<int>& classes, std::vector<float2>* tw, std::vector<double2>* tw64,
                           std::map<int, int>* off) {
  for (int n : classes) {
    (*off)[n] = (int)tw->size();
    rf_twiddles(n, tw);
    rf_twiddles64(n, tw64);
  }
}

}  // namespace wighost
