// Host execution of the adjoint-form kernels (csrc/wig_jit_adjoint.cuh): N forward
// steps as wiga_forward with the per-step records kept (Y_n = K W_n; damped: U_n and
// s_n), then N adjoint steps as wig_step_adjoint from step N - 1 down to 0
// (csrc/wig_adjoint.cu), over the tables wiga_create builds (csrc/wig_adjoint_host.h).
// WIGA_NX, WIGA_NP, WIGA_PW, WIGA_PREC come from the command line.  Test
// infrastructure: tests/test_emu_cpu.py builds it and compares with the torch twin.
//
//   adjoint_emu X_in L_in eps_in W_out lam_out grad_out n_steps amp dt d_theta d_lambda v4 v2 v0 gamma f_eps
//
// X_in / L_in / W_out / lam_out: (WIGA_NP, WIGA_NX) complex64 (WIGA_PREC 0) or complex128
// (WIGA_PREC 1); eps_in: n_steps doubles; grad_out: n_steps x 3 doubles.  hbar = mass = 1.
#include "shim.h"
#include "wig_jit_adjoint.cuh"
#include "wig_batch_host.h"
#include "wig_adjoint_host.h"

#include <cstdlib>

namespace {

// the fields of wiga_desc (include/wigner_b200.h) that adjoint_setup reads
struct Desc {
  int n_x, n_p;
  double x_amplitude, p_amplitude, hbar, mass, dt, d_theta, d_lambda, v4, v2, v0, gamma, f_eps;
};

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
  if (argc != 17) {
    std::fprintf(stderr, "usage: %s X L eps W_out lam_out grad_out n_steps amp dt d_theta d_lambda v4 v2 v0 gamma "
                 "f_eps\n", argv[0]);
    return 2;
  }
  constexpr int nx = WIGA_NX, np = WIGA_NP;
  const long n_steps = std::atol(argv[7]);
  if (n_steps < 1) return 2;
  Desc d{};
  d.n_x = nx; d.n_p = np;
  d.x_amplitude = d.p_amplitude = std::atof(argv[8]);
  d.dt = std::atof(argv[9]); d.d_theta = std::atof(argv[10]); d.d_lambda = std::atof(argv[11]);
  d.v4 = std::atof(argv[12]); d.v2 = std::atof(argv[13]); d.v0 = std::atof(argv[14]);
  d.gamma = std::atof(argv[15]); d.f_eps = std::atof(argv[16]);
  d.hbar = 1.; d.mass = 1.;
  const size_t plane = (size_t)nx * np;
  std::vector<WigaC> W(plane), lam(plane), Y((size_t)n_steps * plane), U((size_t)n_steps * plane);
  std::vector<double> eps(n_steps), grad(3 * n_steps, 0.);
  std::vector<double2> s(n_steps);
  if (!read_all(argv[1], W.data(), plane) || !read_all(argv[2], lam.data(), plane) ||
      !read_all(argv[3], eps.data(), (size_t)n_steps))
    return 4;

  // wiga_create
  wig::AArgs a{};
  wighost::AdjTables t;
  wighost::adjoint_setup(d, a, &t);
#if WIGA_PREC == 1
  std::vector<double2> twx, twp;
  wighost::rf_twiddles64(nx, &twx);
  wighost::rf_twiddles64(np, &twp);
#else
  std::vector<float2> twx, twp;
  wighost::rf_twiddles(nx, &twx);
  wighost::rf_twiddles(np, &twp);
#endif
  std::vector<double2> sc = {make_double2(1., 0.), make_double2(1., 0.), make_double2(0., 0.)};
  a.tw_x = twx.data(); a.tw_p = twp.data();
  a.rtab = t.rtab.data(); a.mm = t.mm.data(); a.rth = t.rth.data(); a.sfp = t.sfp.data(); a.ths = t.ths.data();
  a.pend = sc.data(); a.coef = sc.data() + 1;
  const int spw_x = wig::rf_spw(nx), spw_p = wig::rf_spw(np), ct = WIGA_PW * spw_p;
  const int grid_x = np / spw_x, grid_p = nx / ct, grid_d = 3;
  std::vector<double> part(3 * (grid_p > grid_d ? grid_p : grid_d));
  // wiga_create's dynamic shared memory
  const size_t smem_x = (size_t)spw_x * (nx + (wig::rf_g(nx) == 8 ? 8 : 0)) * sizeof(WigaC);
  const size_t smem_p = (size_t)2 * ct * np * sizeof(WigaC);
  const bool damped = a.damped != 0;

  // wiga_forward with the records kept
  for (long n = 0; n < n_steps; ++n) {
    WigaC* Yn = Y.data() + (size_t)n * plane;
    WigaC* Un = damped ? U.data() + (size_t)n * plane : nullptr;
    const WigaC* Wc = W.data();
    const int use_pend = (damped && n > 0) ? 1 : 0;
    emu_launch(grid_x, 32, [&] { wiga_xpass(a, Wc, Yn, 1., use_pend); }, smem_x);
    emu_launch(grid_p, WIGA_PW * 32, [&] { wiga_ppass(a, Yn, W.data(), Un, eps.data(), (long long)n, part.data()); },
               smem_p);
    if (damped) emu_launch(1, 32, [&] { wiga_fwd_finalize(a, part.data(), grid_p, s.data(), (long long)n); });
  }
  if (damped) {
    emu_launch(4, 256, [&] { wiga_scale(a, W.data(), (long long)plane); });
    emu_launch(1, 32, [&] { wiga_reset_pend(a); });
  }
  // wig_step_adjoint from the last step down
  for (long n = n_steps - 1; n >= 0; --n) {
    const WigaC* Yn = Y.data() + (size_t)n * plane;
    if (damped) {
      const WigaC* Un = U.data() + (size_t)n * plane;
      emu_launch(grid_d, 256, [&] { wiga_dot(lam.data(), Un, (long long)plane, part.data()); });
      emu_launch(1, 32, [&] { wiga_adj_coef(a, part.data(), grid_d, s.data(), (long long)n); });
    }
    emu_launch(grid_p, WIGA_PW * 32,
               [&] { wiga_ppass_T(a, lam.data(), Yn, eps.data(), (long long)n, part.data()); }, smem_p);
    emu_launch(1, 32, [&] { wiga_grad_finalize(part.data(), grid_p, grad.data(), (long long)n); });
    const WigaC* lc = lam.data();
    emu_launch(grid_x, 32, [&] { wiga_xpass(a, lc, lam.data(), -1., 0); }, smem_x);
  }
  if (!write_all(argv[4], W.data(), plane) || !write_all(argv[5], lam.data(), plane) ||
      !write_all(argv[6], grad.data(), grad.size()))
    return 4;
  return 0;
}
