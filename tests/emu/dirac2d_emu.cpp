// Host execution of the Dirac2D kernels (csrc/wig_jit_dirac.cuh) in the launch
// sequence of dirac_run (csrc/wig_capi.cu: dirac_run_begin / _step / _end),
// with the tile macros DIR_* given on the command line.  Test infrastructure:
// tests/test_emu_cpu.py builds it and compares the result with the oracle.
//
//   dirac2d_emu psi_in psi_out obs_out n_steps x_amplitude y_amplitude dt mass c
//
// psi_in / psi_out: (4, DIR_NY, DIR_NX) complex128; obs_out: n_steps x 10
// doubles.  Constants are used exactly (no '%f' rounding).  The potentials are
// fixed here and restated by the test for the oracle.
#include "shim.h"

struct UserPhys {
  double cf[8];
  double A0(double t, double x, double y) const { return -1. / sqrt(x * x + y * y + 0.5) + 0.3 * t * x; }
  double A1(double, double, double y) const { return -0.5 * y; }
  double A2(double, double x, double) const { return 0.5 * x; }
  double A3(double, double, double) const { return 0.; }
};

#include "wig_jit_dirac.cuh"

#include <cstdlib>

namespace {

// the host tables of dirac_create: shifted coordinate ranges, twiddles in extended precision
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

}  // namespace

int main(int argc, char** argv) {
  if (argc != 10) {
    std::fprintf(stderr, "usage: %s psi_in psi_out obs_out n_steps x_amp y_amp dt mass c\n", argv[0]);
    return 2;
  }
  constexpr int NX = DIR_NX, NY = DIR_NY;
  const long n_steps = std::atol(argv[4]);
  const double xa = std::atof(argv[5]), ya = std::atof(argv[6]), dt = std::atof(argv[7]);
  const double mass = std::atof(argv[8]), c = std::atof(argv[9]);
  if (n_steps < 1 || NY % DIR_ROWS != 0 || NX % DIR_C != 0) return 2;
  const size_t npts = 4ull * NX * NY;
  std::vector<double2> psi(npts);
  if (!read_all(argv[1], psi.data(), npts * sizeof(double2))) return 4;

  // GPU_Dirac2D.py:312-346
  const double dX = 2. * xa / NX, dY = 2. * ya / NY;
  const double Pxa = M_PI / dX, Pya = M_PI / dY;
  const double dPx = 2. * Pxa / NX, dPy = 2. * Pya / NY;
  const int n_row = NY / DIR_ROWS, n_col = NX / DIR_C;
  // dirac_plan's dynamic shared memory
  const size_t sm_row = (size_t)wig::padded_size(4 * DIR_ROWS * NX) * sizeof(double2);
  const size_t sm_col = (size_t)wig::padded_size(4 * DIR_C * NY) * sizeof(double2);

  std::vector<double> xt = shifted_range(xa, NX), yt = shifted_range(ya, NY);
  std::vector<double> pxt = shifted_range(Pxa, NX), pyt = shifted_range(Pya, NY);
  std::vector<double> bx(2 * NX), by(2 * NY);
  std::vector<double2> twx = twiddles(NX), twy = twiddles(NY);
  std::vector<double> pr0((size_t)n_row * wig::DNR), pr1((size_t)n_row * wig::DNR), pc((size_t)n_col * wig::DNC);
  std::vector<double> obs((size_t)n_steps * wig::DNOBS, 0.);
  double2 scale{1., 0.};

  emu_launch(1, 64, [&] { dirac_setup(bx.data(), by.data()); });

  wig::DiracArgs a{};
  a.mass = mass; a.c = c; a.dt = dt; a.dX = dX; a.dY = dY; a.dPx = dPx; a.dPy = dPy;
  a.dX_e = dX; a.dY_e = dY; a.dPx_e = dPx; a.dPy_e = dPy; a.mass_e = mass; a.c_e = c;
  a.x_tab = xt.data(); a.y_tab = yt.data(); a.px_tab = pxt.data(); a.py_tab = pyt.data();
  a.bx = bx.data(); a.by = by.data(); a.tw_x = twx.data(); a.tw_y = twy.data();
  a.part_row[0] = pr0.data(); a.part_row[1] = pr1.data(); a.part_col = pc.data();
  a.n_row_cta = n_row; a.n_col_cta = n_col;

  double2* P = psi.data();
  // dirac_run_begin: first row pass (x sums, row FFT)
  {
    const double t_obs = dt * 1.;
    emu_launch(n_row, DIR_RNT, [&] { dirac_rowpass(a, P, 0, 0, 0., t_obs, nullptr); }, sm_row);
  }
  // dirac_run_step
  for (long n = 0; n < n_steps; ++n) {
    emu_launch(n_col, DIR_CNT, [&] { dirac_colpass(a, P); }, sm_col);
    const int mode = (n == n_steps - 1) ? 2 : 1, parity = (int)((n + 1) & 1);
    const double t_step = dt * (double)(n + 1), t_obs = dt * (double)(n + 2);
    double* orow = obs.data() + (size_t)n * wig::DNOBS;
    emu_launch(n_row, DIR_RNT, [&] { dirac_rowpass(a, P, mode, parity, t_step, t_obs, orow); }, sm_row);
  }
  // dirac_run_end: the final Normalize_X factor and its application
  {
    const int parity = (int)(n_steps & 1);
    emu_launch(1, DIR_SNT, [&] { dirac_final(a, parity, &scale); });
    const long n = (long)npts;
    emu_launch(2, DIR_SNT, [&] { dirac_scale(P, n, &scale); });
  }
  if (!write_all(argv[2], psi.data(), npts * sizeof(double2))) return 4;
  if (!write_all(argv[3], obs.data(), obs.size() * sizeof(double))) return 4;
  return 0;
}
