// Host execution of the Dirac3D kernels (csrc/wig_jit_dirac3.cuh) in the launch
// sequence of dirac3_run (csrc/wig_dirac3.cu), with the tile macros D3_* given
// on the command line.  Test infrastructure: tests/test_emu_cpu.py builds it
// and compares the result with the oracle.
//
//   dirac3d_emu psi_in psi_out obs_out n_steps x_amp y_amp z_amp dt mass c max_cta
//
// psi_in / psi_out: (4, D3_NZ, D3_NY, D3_NX) complex128; obs_out: n_steps x 12
// doubles.  hbar = 1, constants used exactly.  max_cta caps every pass's grid
// (the passes are grid-stride), so that CTAs take several tiles.  The
// potentials are fixed here and restated by the test for the oracle.
#include "shim.h"

struct UserPhys {
  double cf[8];
  double A0(double t, double x, double y, double z) const {
    return -1. / sqrt(x * x + y * y + z * z + 0.5) + 0.2 * t * z;
  }
  double A1(double, double, double y, double) const { return -0.5 * y; }
  double A2(double, double x, double, double) const { return 0.5 * x; }
  double A3(double, double, double, double z) const { return 0.1 * z; }
};

#include "wig_jit_dirac3.cuh"

namespace {

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
  if (argc != 12) {
    std::fprintf(stderr, "usage: %s psi_in psi_out obs_out n_steps x_amp y_amp z_amp dt mass c max_cta\n", argv[0]);
    return 2;
  }
  constexpr int NX = D3_NX, NY = D3_NY, NZ = D3_NZ;
  const long n_steps = std::atol(argv[4]);
  const double xa = std::atof(argv[5]), ya = std::atof(argv[6]), za = std::atof(argv[7]);
  const double dt = std::atof(argv[8]), mass = std::atof(argv[9]), c = std::atof(argv[10]);
  const int max_cta = std::atoi(argv[11]);
  if (n_steps < 1 || max_cta < 1) return 2;
  const size_t npts = 4ull * NX * NY * NZ;
  std::vector<double2> psi(npts);
  if (!read_all(argv[1], psi.data(), npts * sizeof(double2))) return 4;

  // d3_plan / dirac3_create (GPU_Dirac3D.py:637-683)
  const double dX = 2. * xa / NX, dY = 2. * ya / NY, dZ = 2. * za / NZ;
  const double dPx = 2 * (M_PI / dX) / NX, dPy = 2 * (M_PI / dY) / NY, dPz = 2 * (M_PI / dZ) / NZ;
  const int gx = clampi(NY * NZ / D3_ROWS, 1, max_cta);
  const int gy = clampi(4 * NZ * (NX / D3_YC), 1, max_cta);
  const int gz = clampi(NY * (NX / D3_ZC), 1, max_cta);
  const int gn = clampi((int)(npts / (4L * D3_SNT)), 1, max_cta);
  // dirac3_plan's dynamic shared memory
  const size_t sm_x = (size_t)wig::padded_size(4 * D3_ROWS * NX) * sizeof(double2);
  const size_t sm_y = (size_t)wig::padded_size(NY * D3_YC) * sizeof(double2);
  const size_t sm_z = (size_t)wig::padded_size(4 * D3_ZC * NZ) * sizeof(double2);

  wig::Dirac3Args a{};
  a.hbar = 1.; a.mass = mass; a.c = c; a.dt = dt;
  a.dX = dX; a.dY = dY; a.dZ = dZ; a.dPx = dPx; a.dPy = dPy; a.dPz = dPz;
  a.dX_e = dX; a.dY_e = dY; a.dZ_e = dZ; a.dPx_e = dPx; a.dPy_e = dPy; a.dPz_e = dPz;
  std::vector<double2> twx = twiddles(NX), twy = twiddles(NY), twz = twiddles(NZ);
  const size_t npart_x = (size_t)(gx * wig::D3X > gn ? gx * wig::D3X : gn);
  std::vector<double> px0(npart_x), px1(npart_x), pp((size_t)gz * wig::D3P);
  std::vector<double> sc = {1.0, 0.0};   // scale, s1
  std::vector<double> obs((size_t)n_steps * wig::D3NOBS, 0.);
  a.tw_x = twx.data(); a.tw_y = twy.data(); a.tw_z = twz.data();
  a.part_x[0] = px0.data(); a.part_x[1] = px1.data(); a.part_p = pp.data();
  a.scale = sc.data(); a.s1 = sc.data() + 1;
  a.n_x_cta = gx; a.n_z_cta = gz;

  double2* P = psi.data();
  // Normalize_GPU before the loop (:1323)
  {
    const long n = (long)npts;
    emu_launch(gn, D3_SNT, [&] { d3_norm(a, P, n); });
    emu_launch(1, D3_SNT, [&] { d3_norm_fin(a, gn); });
  }
  emu_launch(gx, D3_XNT, [&] { d3_xpass(a, P, 0, 0, 1, 0., dt, 0, nullptr); }, sm_x);
  for (long k = 1; k <= n_steps; ++k) {
    emu_launch(gy, D3_YNT, [&] { d3_ypass_fwd(a, P); }, sm_y);
    emu_launch(gz, D3_ZNT, [&] { d3_zpass(a, P); }, sm_z);
    emu_launch(gy, D3_YNT, [&] { d3_ypass_inv(a, P); }, sm_y);
    const int mode = (k == n_steps) ? 2 : 1, parity = (int)(k & 1);
    const double tA = dt * (double)k, tobs = dt * (double)(k + 1);
    double* oprev = obs.data() + (size_t)(k - 1) * wig::D3NOBS;
    emu_launch(gx, D3_XNT, [&] { d3_xpass(a, P, mode, parity, 0, tA, tobs, (long long)k, oprev); }, sm_x);
  }
  if (!write_all(argv[2], psi.data(), npts * sizeof(double2))) return 4;
  if (!write_all(argv[3], obs.data(), obs.size() * sizeof(double))) return 4;
  return 0;
}
