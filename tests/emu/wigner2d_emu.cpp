// Host execution of the complex128 Wigner2D kernels (csrc/wig_jit_wigner.cuh)
// in the launch sequence of wig_run for a plan with Caldeira-Leggett (WIG_DAMP 1)
// or first-order ODM Lindblad damping (WIG_DAMP 0; odm 1: one term, 2: the two
// terms of GPU_Wigner2D_ODM2), Lie-split or, with
// WIG_STRANG 1, the Strang / Gross-Pitaevskii step (csrc/wig_capi.cu:
// wig_run_begin / wig_run_step / wig_run_step_strang / wig_run_end), with the
// tile macros WIG_* given on the command line.  Test infrastructure:
// tests/test_emu_cpu.py builds it and compares the result with the oracle.
//
//   wigner2d_emu W_in W_out obs_out n_prop x_amp p_amp dt gamma d_theta d_lambda odm a_gp
//                [bloch_steps dtb W0_in|-]
//
// W_in / W_out: (WIG_NP, WIG_NX) complex128; obs_out: (n_prop + 1) x 11
// doubles, then (Strang) n_prop values of sum P(x)^2 dx.  With bloch_steps > 0
// (WIG_STRANG 1) it makes that many imaginary-time steps of dtb instead, as
// wig_bloch_step (t_index = step, W0 optional), and obs_out holds their
// WIG_BLOCH_NSTATS = 10 numbers each.  hbar = mass = 1, constants used exactly.
// The expressions are fixed here and restated by the test for the oracle.
#include "shim.h"

#define __constant__
double dt, dx, dp, dtheta, dlambda, mass, hBar, D_Theta, D_Lambda;

struct UserPhys {
  double cf[8];
  double Potential(double t, double x) const { return 0.05 * pow(x, 4) - pow(x, 2) + 0.2 * x * sin(3. * t); }
  double KineticEnergy(double p) const { return 0.5 * p * p; }
  double f(double p) const { return fabs(p); }
  double DPotential(double t, double x) const { return 0.2 * pow(x, 3) - 2. * x + 0.2 * sin(3. * t); }
};

#include "wig_jit_wigner.cuh"
#include "wig_batch_host.h"   // register-FFT twiddle tables

namespace {

std::vector<double> shifted_range(double amp, int n) {
  const double d = 2. * amp / (double)n;
  const double start = -amp, stop = amp - d;
  const double step = (stop - start) / (double)(n - 1);
  std::vector<double> y(n), out(n);
  for (int i = 0; i < n; ++i) y[i] = (double)i * step + start;
  y[n - 1] = stop;
  for (int k = 0; k < n; ++k) out[k] = y[(k + n / 2) % n];
  return out;
}

std::vector<double2> twiddles(int n) {
  const long double pi = 3.141592653589793238462643383279502884L;
  std::vector<double2> t(n);
  for (int m = 0; m < n; ++m) {
    const long double a = 2.0L * pi * (long double)m / (long double)n;
    double c = (double)cosl(a), s = (double)(-sinl(a));
    if (fabs(c) < 1e-18) c = 0.;
    if (fabs(s) < 1e-18) s = 0.;
    t[m] = make_double2(c, s);
  }
  return t;
}

bool read_all(const char* path, void* p, size_t bytes) {
  FILE* f = std::fopen(path, "rb");
  if (!f) return false;
  const bool ok = std::fread(p, 1, bytes, f) == bytes;
  std::fclose(f);
  return ok;
}

bool write_all(const char* path, const void* p, size_t bytes) {
  FILE* f = std::fopen(path, "wb");
  if (!f) return false;
  const bool ok = std::fwrite(p, 1, bytes, f) == bytes;
  std::fclose(f);
  return ok;
}

int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

}  // namespace

int main(int argc, char** argv) {
  if (argc != 13 && argc != 16) {
    std::fprintf(stderr, "usage: %s W_in W_out obs_out n_prop x_amp p_amp dt gamma d_theta d_lambda odm a_gp "
                 "[bloch_steps dtb W0_in|-]\n", argv[0]);
    return 2;
  }
  const long bloch_steps = argc == 16 ? std::atol(argv[13]) : 0;
  constexpr int NX = WIG_NX, NP = WIG_NP, NOBS = 11;
  const long n_prop = std::atol(argv[4]);
  const double xa = std::atof(argv[5]), pa = std::atof(argv[6]);
  const double gamma = std::atof(argv[8]);
  const int odm = std::atoi(argv[11]);
  const double a_gp = std::atof(argv[12]);
  // WIG_DAMP 1: Caldeira-Leggett; 0: ODM damping (odm 1, 2) or none (gamma 0)
  if (n_prop < 1 || NP % WIG_XROWS != 0 || NX % WIG_PC != 0 || (odm != 0 && WIG_DAMP != 0) ||
      (odm == 0 && WIG_DAMP == 0 && gamma != 0.))
    return 2;
  dt = std::atof(argv[7]);
  D_Theta = std::atof(argv[9]);
  D_Lambda = std::atof(argv[10]);
  mass = hBar = 1.;
  const size_t npts = (size_t)NX * NP;
  std::vector<double2> W(npts);
  if (!read_all(argv[1], W.data(), npts * sizeof(double2))) return 4;

  // wig_plan / wig_create
  dx = 2. * xa / NX;
  dp = 2. * pa / NP;
  dtheta = 2. * M_PI / (2. * pa);
  dlambda = 2. * M_PI / (2. * xa);
  const int n_cta_x = NP / WIG_XROWS, n_cta_p = NX / WIG_PC;
  // wig_plan's dynamic shared memory
  const size_t tile_x = (size_t)wig::padded_size(WIG_XROWS * NX) * sizeof(double2);
  const size_t tile_p = (size_t)wig::padded_size(WIG_PC * NP) * sizeof(double2);
  const size_t sm_x = tile_x, sm_p = WIG_DAMP == 1 ? 2 * tile_p + 2 * NP * sizeof(double) : tile_p;
  const size_t sm_ox = 2 * tile_x, sm_op = 2 * tile_p, sm_ph = tile_p;
  const size_t sm_gph = ((size_t)wig::padded_size(NX) + wig::padded_size(WIG_XROWS * NX)) * sizeof(double2);
  const int n_cta_r = clampi(NX * NP / (4 * WIG_RNT), 1, 296);
#if WIG_RF
  // the register-FFT passes (wig_plan's rf branch)
  const int rf_gx = NP / (WIG_RFXW * wig::rf_spw(NX)), rf_gp = NX / (WIG_RFPW * wig::rf_spw(NP));
  const size_t sm_rx = (size_t)WIG_RFXW * wig::rf_spw(NX) * (NX + (wig::rf_g(NX) == 8 ? 8 : 0)) * sizeof(double2);
  const size_t sm_rp = (size_t)(WIG_DAMP == 1 ? 2 : 1) * WIG_RFPW * wig::rf_spw(NP) * NP * sizeof(double2) + 1024;
  const wig::TensorMap no_map{};   // the thread-load path of the emulation takes no tensor map
  std::vector<double2> rtwx, rtwp;
  wighost::rf_twiddles64(NX, &rtwx);
  wighost::rf_twiddles64(NP, &rtwp);
#else
  const int rf_gx = 1, rf_gp = 1;
#endif

  wig::WigArgs a{};
  a.dt = dt; a.dx = dx; a.dp = dp; a.dtheta = dtheta; a.dlambda = dlambda; a.mass = mass; a.hbar = hBar;
  a.D_theta = D_Theta; a.D_lambda = D_Lambda;
  a.dX = dx; a.dP = dp; a.mass_exact = mass;
  {
    const double g = dt * gamma;
    const double c1 = 2. / 3. * g, c2 = 2. / 2. * g, c3 = 2. * g;
    const double k1 = (c1 + c2) != 0. ? c1 * c2 / (c1 + c2) : 0.;
    a.cl_k1 = make_double2(0., k1);
    a.cl_k12 = make_double2(0., c1 + c2);
    a.cl_c3 = make_double2(0., c3);
  }
  std::vector<double> xt = shifted_range(xa, NX), pt = shifted_range(pa, NP);
  std::vector<double> tht = shifted_range(dtheta * NP / 2., NP), ths(NP);
  for (int i = 0; i < NP; ++i) ths[i] = tht[i] * (1.0 / (double)NP);
  std::vector<double> lt = shifted_range(dlambda * NX / 2., NX);
  const UserPhys ph{};
  std::vector<double> dv(NX), v0(NX);
  for (int k = 0; k < NX; ++k) {
    dv[k] = ph.DPotential(0., xt[k]);
    v0[k] = ph.Potential(0., xt[k]);
  }
  std::vector<double2> twx = twiddles(NX), twp = twiddles(NP);
  std::vector<double> rl(NX), rt(NP), m1(NX), m2(NX), sfp(NP), rth(NP);
  const int nparts = std::max(std::max(std::max(n_cta_x, n_cta_p), n_cta_r), std::max(rf_gx, rf_gp));
  std::vector<double> partials((size_t)nparts * wig::NACC, 0.), partials_im(odm ? (size_t)nparts * wig::NIM : 0, 0.);
  std::vector<double> obs((size_t)(n_prop + 1) * NOBS, 0.);
  double2 scale{1., 0.};
  a.x_tab = xt.data(); a.p_tab = pt.data(); a.dV_tab = dv.data(); a.V0_tab = v0.data(); a.theta_s = ths.data();
  a.r_lambda = rl.data(); a.r_theta = rt.data(); a.mask1 = m1.data(); a.mask2s = m2.data(); a.sfp = sfp.data();
  a.tw_x = twx.data(); a.tw_p = twp.data(); a.partials = partials.data(); a.n_partials = 0;
  a.partials_im = odm ? partials_im.data() : nullptr;   // as wig_create: ODM plans only
  a.lambda_tab = lt.data(); a.hbar_exact = hBar; a.L_material = 1.;
  a.r_theta_half = rth.data();
  a.gp_coef = a_gp;
#if WIG_RF
  a.rtw_x = rtwx.data();
  a.rtw_p = rtwp.data();
#endif
  int status = 0;
  a.status = &status;
  emu_launch(1, 64, [&] { wig_setup(a, rl.data(), rt.data(), m1.data(), m2.data(), sfp.data(), rth.data()); });
  // Lindbladian_ODM_Order1: scale dt 2 gamma weight / n_p, five intermediate planes; odm 1: one term
  // (weight 1, sign 1), odm 2: GPU_Wigner2D_ODM2's damping (weight 1, sign 1) then pumping (weight 0.5,
  // sign -1)
  const double odm_w[2] = {1., 0.5}, odm_sign[2] = {1., -1.};
  std::vector<double2> T(odm ? 5 * npts : 0);

  double2* Wp = W.data();
#if WIG_STRANG
  if (bloch_steps > 0) {
    // wig_bloch_step: mean-field exponent, half potential, kinetic, mean-field exponent, half
    // potential, [W -= c W0], normalisation by the complex sum, then the step statistics
    const double dtb = std::atof(argv[14]);
    std::vector<double2> W0;
    if (std::strcmp(argv[15], "-") != 0) {
      W0.resize(npts);
      if (!read_all(argv[15], W0.data(), npts * sizeof(double2))) return 4;
    }
    const double2* W0p = W0.empty() ? nullptr : W0.data();
    const int gp = a_gp != 0., gcnt = NX < 256 ? NX : 256, n_chunks = NP / 16;
    std::vector<double2> chunks((size_t)n_chunks * NX), rows(NP);
    std::vector<double> Px(NX), gexp(npts), bpart((size_t)n_cta_r * wig::NBL), psq(1);
    const long n = (long)npts;
    const int gaxpy = clampi((int)(n / (4 * WIG_RNT)), 1, 592);
    const double dXdP = a.dX * a.dP, pf = 2. * M_PI * hBar * dXdP;
    auto sums = [&](const double2* w0, double* out) {
      emu_launch(n_cta_r, WIG_RNT, [&] { wig_bloch_reduce(a, Wp, w0, bpart.data()); });
      for (int v = 0; v < wig::NBL; ++v) out[v] = 0.;
      for (int c = 0; c < n_cta_r; ++c)
        for (int v = 0; v < wig::NBL; ++v) out[v] += bpart[(size_t)c * wig::NBL + v];
    };
    auto marginal = [&](double* psq_out) {
      emu_launch2d(NX / gcnt, NP / 16, gcnt, [&] { wig_gp_colsum(Wp, chunks.data()); });
      emu_launch(1, 256, [&] { wig_gp_marginal(a, chunks.data(), n_chunks, 0, Px.data(), psq_out); });
    };
    auto exponent = [&]() -> const double* {
      if (!gp) return nullptr;
      marginal(nullptr);
      emu_launch(n_cta_x, WIG_XNT, [&] { wig_gp_bloch(a, Px.data(), dtb, gexp.data()); }, sm_gph);
      return gexp.data();
    };
    std::vector<double> stats((size_t)bloch_steps * 10, 0.);
    for (long k = 0; k < bloch_steps; ++k) {
      const double t = (double)k * dt;
      const double* ge = exponent();
      emu_launch(n_cta_p, WIG_PNT, [&] { wig_bloch_ppass(a, Wp, t, dtb, ge); }, sm_ph);
      emu_launch(n_cta_x, WIG_XNT, [&] { wig_bloch_xpass(a, Wp, dtb); }, sm_x);
      ge = exponent();
      emu_launch(n_cta_p, WIG_PNT, [&] { wig_bloch_ppass(a, Wp, t, dtb, ge); }, sm_ph);
      double sm[wig::NBL];
      if (W0p) {
        sums(W0p, sm);
        const double2 c = make_double2(pf * sm[9], pf * sm[10]), one = make_double2(1., 0.);
        emu_launch(gaxpy, WIG_RNT, [&] { wig_bloch_axpy(Wp, W0p, n, c, one); });
      }
      sums(nullptr, sm);
      const double2 nrm = make_double2(sm[0] * dXdP, sm[1] * dXdP);
      const double2 inv = wig::crecip(nrm), zero = make_double2(0., 0.);
      emu_launch(gaxpy, WIG_RNT, [&] { wig_bloch_axpy(Wp, nullptr, n, zero, inv); });
      double* st = stats.data() + (size_t)k * 10;
      sums(nullptr, sm);
      for (int q = 0; q < 5; ++q) st[q] = dXdP * sm[2 + q];
      st[5] = pf * sm[7];
      st[6] = pf * sm[8];
      if (gp) {
        marginal(psq.data());
        st[7] = 0.5 * a_gp * psq[0];
      }
      if (W0p) {
        emu_launch(NP, 256, [&] { wig_rowsum(Wp, rows.data()); });
        for (const double2& r : rows)
          if (r.x * a.dX < 0.) { st[8] = 1.; break; }
      }
      st[9] = nrm.x;
    }
    if (!write_all(argv[2], W.data(), npts * sizeof(double2))) return 4;
    if (!write_all(argv[3], stats.data(), stats.size() * sizeof(double))) return 4;
    return 0;
  }
#endif
  // wig_run_begin: partial sums of W for the initial normalisation and sample 0
  emu_launch(n_cta_r, WIG_RNT, [&] { wig_reduce(a, Wp); });
  a.n_partials = n_cta_r;
  // wig_run_step (first call of a run: normalise on load; damped steps renormalise)
  const bool damped = gamma != 0.;
#if WIG_STRANG
  // wig_gp_terms: column sums over 16-row chunks, the marginal, the per-row phase
  const int gp = a_gp != 0.;
  const int gcnt = NX < 256 ? NX : 256, n_chunks = NP / 16;
  std::vector<double2> chunks((size_t)n_chunks * NX);
  std::vector<double> Px(NX), phase(npts), psq(n_prop, 0.);
  auto gp_terms = [&](int scale_mode, double* psq_out) {
    emu_launch2d(NX / gcnt, NP / 16, gcnt, [&] { wig_gp_colsum(Wp, chunks.data()); });
    emu_launch(1, 256, [&] { wig_gp_marginal(a, chunks.data(), n_chunks, scale_mode, Px.data(), psq_out); });
    emu_launch(n_cta_x, WIG_XNT, [&] { wig_gp_phase(a, Px.data(), phase.data()); }, sm_gph);
  };
  const double* gph = gp ? phase.data() : nullptr;
#endif
  for (long n = 0; n < n_prop; ++n) {
    const int mode = (n == 0) ? 1 : (damped ? 2 : 0);
    double* orow = obs.data() + (size_t)n * NOBS;
    const double t = (double)n * dt;
#if WIG_STRANG
    if (gp) gp_terms(mode, nullptr);
    emu_launch(n_cta_p, WIG_PNT, [&] { wig_ppass_half(a, Wp, t, mode, orow, gph); }, sm_ph);
    emu_launch(n_cta_x, WIG_XNT, [&] { wig_xpass(a, Wp, 0, nullptr); }, sm_x);
    if (gp) gp_terms(0, psq.data() + n);
    emu_launch(n_cta_p, WIG_PNT, [&] { wig_ppass_half_final(a, Wp, t, gph); }, sm_p);
#elif WIG_RF
    emu_launch(rf_gx, WIG_RFXW * 32, [&] { wig_xpass_rf(a, Wp, mode, orow); }, sm_rx);
    emu_launch(rf_gp, WIG_RFPW * 32, [&] { wig_ppass_rf(a, Wp, t, no_map); }, sm_rp);
#else
    emu_launch(n_cta_x, WIG_XNT, [&] { wig_xpass(a, Wp, mode, orow); }, sm_x);
    emu_launch(n_cta_p, WIG_PNT, [&] { wig_ppass(a, Wp, t); }, sm_p);
#endif
    for (int j = 0; j < odm; ++j) {
      const double coef = dt * 2 * gamma * odm_w[j] / 1. * (1.0 / (double)NP), sign = odm_sign[j];
      emu_launch(n_cta_x, WIG_XNT, [&] { wig_odm_xpass(a, Wp, T.data()); }, sm_ox);
      emu_launch(n_cta_p, WIG_PNT, [&] { wig_odm_ppass(a, Wp, T.data(), coef, sign); }, sm_op);
    }
    a.n_partials = WIG_RF ? rf_gp : n_cta_p;
  }
  // wig_run_end
  {
    const int fmode = damped ? 2 : 0;
    double* last = obs.data() + (size_t)n_prop * NOBS;
    emu_launch(1, WIG_RNT, [&] { wig_finalize(a, fmode, last, &scale); });
    if (fmode != 0) {
      const long n = (long)npts;
      emu_launch(2, WIG_RNT, [&] { wig_scale(Wp, n, &scale); });
    }
  }
  if (!write_all(argv[2], W.data(), npts * sizeof(double2))) return 4;
#if WIG_STRANG
  obs.insert(obs.end(), psq.begin(), psq.end());
#endif
  if (!write_all(argv[3], obs.data(), obs.size() * sizeof(double))) return 4;
  return 0;
}
