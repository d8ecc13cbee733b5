// Host-side set-up of the adjoint form (wiga_create): constants and factor
// tables of one grid.  Included by the library (wig_adjoint.cu) and by the
// host execution of the device code (tests/emu/adjoint_emu.cpp).
#pragma once
#include <math.h>

#include <vector>

#include "wig_adjoint.cuh"

namespace wighost {

struct AdjTables {
  std::vector<double> rtab, mm, rth, sfp, ths;
};

// D: any struct with the fields of wiga_desc.  Fills the scalar fields of a
// (pointers are set by the caller) and the tables (expPLambda_source :153,
// expPotential_source :117-123, theta_fp_source :422-428 of GPU_Wigner2D_FFT.py).
template <class D>
void adjoint_setup(const D& d, wig::AArgs& a, AdjTables* t) {
  const int nx = d.n_x, np = d.n_p;
  a.n_x = nx;
  a.n_p = np;
  a.damped = d.gamma != 0. ? 1 : 0;
  a.dt = d.dt;
  a.hbar = d.hbar;
  a.mass = d.mass;
  a.dx = 2. * d.x_amplitude / nx;
  a.dp = 2. * d.p_amplitude / np;
  a.dtheta = 2. * M_PI / (2. * d.p_amplitude);
  a.dlambda = 2. * M_PI / (2. * d.x_amplitude);
  a.v4 = d.v4;
  a.v2 = d.v2;
  a.v0 = d.v0;
  // CaldeiraDissipatorOrder3 (GPU_Wigner2D_FFT.py:1145-1157) in Horner form: imaginary parts
  const double g = d.dt * d.gamma, c1 = 2. / 3. * g, c2 = g, c3 = 2. * g;
  a.cl1 = (c1 + c2) != 0. ? c1 * c2 / (c1 + c2) : 0.;
  a.cl2 = c1 + c2;
  a.cl3 = c3;
  t->rtab.resize(nx);
  t->mm.resize(nx);
  t->rth.resize(np);
  t->sfp.resize(np);
  t->ths.resize(np);
  const double x_max = a.dx * (nx - 1.) / 2., w2 = (10. * a.dx) * (10. * a.dx);
  for (int k = 0; k < nx; ++k) {
    const double j = ((k + nx / 2) % nx) - 0.5 * nx;
    const double lam = a.dlambda * j, x = a.dx * j;
    t->rtab[k] = exp(-d.d_lambda * lam * lam) / (double)nx;
    const double m1 = 1. - exp(-(x - x_max) * (x - x_max) / w2), m2 = 1. - exp(-(x + x_max) * (x + x_max) / w2);
    t->mm[k] = m1 * m2 / (double)np;
  }
  for (int k = 0; k < np; ++k) {
    const double j = ((k + np / 2) % np) - 0.5 * np;
    const double th = a.dtheta * j, p = a.dp * j;
    t->rth[k] = exp(-d.d_theta * th * th * d.dt);
    t->ths[k] = th / (double)np;
    const double f = d.f_eps == 0. ? fabs(p) : p * p / sqrt(p * p + d.f_eps);
    t->sfp[k] = p >= 0. ? f : -f;
  }
}

// p-pass tile: 4 columns (32- or 64-byte row segments)
inline int adjoint_p_warps(int n_p) { return 4 / wig::rf_spw(n_p) > 0 ? 4 / wig::rf_spw(n_p) : 1; }

}  // namespace wighost
