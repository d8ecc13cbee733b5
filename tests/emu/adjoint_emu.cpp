// Host execution of the adjoint-form kernels (csrc/wig_jit_adjoint.cuh): N forward
// steps as wiga_forward with the per-step Y = K W kept, then N adjoint steps as
// wig_step_adjoint from step N - 1 down to 0 (csrc/wig_adjoint.cu).  WIGA_NX,
// WIGA_NP, WIGA_PW come from the command line.  Test infrastructure:
// tests/test_emu_cpu.py builds it and compares with the torch twin.
//
//   adjoint_emu X_in L_in eps_in W_out lam_out grad_out n_steps amp dt d_theta d_lambda v4 v2 v0
//
// X_in / L_in / W_out / lam_out: (WIGA_NP, WIGA_NX) complex64; eps_in / grad_out: n_steps doubles.
// hbar = mass = 1.
#include "shim.h"
#include "wig_jit_adjoint.cuh"

#include <cstdlib>

namespace {

float2 twiddle_f(int n, long long m) {
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

void rf_twiddles(int n, std::vector<float2>* tw) {
  const int E = wig::rf_e(n), G = wig::rf_g(n), Q = E / G;
  for (int a = 0; a < E; ++a)
    for (int g = 0; g < G; ++g) tw->push_back(twiddle_f(n, (long long)g * a));
  for (int i = 0; i < Q; ++i)
    for (int b = 0; b < G; ++b)
      for (int t = 0; t < G; ++t) tw->push_back(twiddle_f(n, (long long)b * (t * Q + i)));
}

template <class T>
bool read_all(const char* path, T* p, size_t n) {
  FILE* f = std::fopen(path, "rb");
  if (!f) return false;
  const bool ok = std::fread(p, sizeof(T), n, f) == n;
  std::fclose(f);
  return ok;
}

template <class T>
bool write_all(const char* path, const T* p, size_t n) {
  FILE* f = std::fopen(path, "wb");
  if (!f) return false;
  const bool ok = std::fwrite(p, sizeof(T), n, f) == n;
  std::fclose(f);
  return ok;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc != 15) {
    std::fprintf(stderr, "usage: %s X L eps W_out lam_out grad_out n_steps amp dt d_theta d_lambda v4 v2 v0\n",
                 argv[0]);
    return 2;
  }
  constexpr int nx = WIGA_NX, np = WIGA_NP;
  const long n_steps = std::atol(argv[7]);
  const double amp = std::atof(argv[8]), dt = std::atof(argv[9]), d_theta = std::atof(argv[10]);
  const double d_lambda = std::atof(argv[11]);
  if (n_steps < 1) return 2;
  const size_t plane = (size_t)nx * np;
  std::vector<float2> W(plane), lam(plane), Y((size_t)n_steps * plane);
  std::vector<double> eps(n_steps), grad(n_steps, 0.);
  if (!read_all(argv[1], W.data(), plane) || !read_all(argv[2], lam.data(), plane) ||
      !read_all(argv[3], eps.data(), (size_t)n_steps))
    return 4;

  // wiga_create
  wig::AArgs a{};
  a.n_x = nx; a.n_p = np;
  a.dt = dt; a.hbar = 1.; a.mass = 1.;
  a.dx = 2. * amp / nx; a.dp = 2. * amp / np;
  a.dtheta = a.dlambda = 2. * M_PI / (2. * amp);
  a.v4 = std::atof(argv[12]); a.v2 = std::atof(argv[13]); a.v0 = std::atof(argv[14]);
  std::vector<float2> twx, twp;
  rf_twiddles(nx, &twx);
  rf_twiddles(np, &twp);
  std::vector<float> rtab(nx), mm(nx), rth(np);
  const double x_max = a.dx * (nx - 1.) / 2., w2 = (10. * a.dx) * (10. * a.dx);
  for (int k = 0; k < nx; ++k) {
    const double j = ((k + nx / 2) % nx) - 0.5 * nx;
    const double lmb = a.dlambda * j, x = a.dx * j;
    rtab[k] = (float)(exp(-d_lambda * lmb * lmb) / (double)nx);
    const double m1 = 1. - exp(-(x - x_max) * (x - x_max) / w2), m2 = 1. - exp(-(x + x_max) * (x + x_max) / w2);
    mm[k] = (float)(m1 * m2 / (double)np);
  }
  for (int k = 0; k < np; ++k) {
    const double th = a.dtheta * (((k + np / 2) % np) - 0.5 * np);
    rth[k] = (float)exp(-d_theta * th * th * dt);
  }
  a.tw_x = twx.data(); a.tw_p = twp.data(); a.rtab = rtab.data(); a.mm = mm.data(); a.rth = rth.data();
  const int spw_x = wig::rf_spw(nx), spw_p = wig::rf_spw(np), ct = WIGA_PW * spw_p;
  const int grid_x = np / spw_x, grid_p = nx / ct;
  std::vector<double> partials(grid_p);

  // wiga_forward with Y kept per step
  for (long n = 0; n < n_steps; ++n) {
    float2* Yn = Y.data() + (size_t)n * plane;
    const float2* Wc = W.data();
    emu_launch(grid_x, 32, [&] { wiga_xpass(a, Wc, Yn, 1.f); });
    emu_launch(grid_p, WIGA_PW * 32, [&] { wiga_ppass(a, Yn, W.data(), eps.data(), (long long)n); });
  }
  // wig_step_adjoint from the last step down
  for (long n = n_steps - 1; n >= 0; --n) {
    const float2* Yn = Y.data() + (size_t)n * plane;
    emu_launch(grid_p, WIGA_PW * 32,
               [&] { wiga_ppass_T(a, lam.data(), Yn, eps.data(), (long long)n, partials.data()); });
    emu_launch(1, 32, [&] { wiga_grad_finalize(partials.data(), grid_p, grad.data(), (long long)n); });
    const float2* lc = lam.data();
    emu_launch(grid_x, 32, [&] { wiga_xpass(a, lc, lam.data(), -1.f); });
  }
  if (!write_all(argv[4], W.data(), plane) || !write_all(argv[5], lam.data(), plane) ||
      !write_all(argv[6], grad.data(), (size_t)n_steps))
    return 4;
  return 0;
}
