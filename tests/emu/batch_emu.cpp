// Host execution of the batched FP32 Wigner2D kernels (csrc/wig_jit_batch.cuh)
// in the launch sequence of wigb_run (csrc/wig_capi.cu: wigb_launch_run), over
// the work lists and tables wigb_create / wigb_set_warps build.  WIGB_WARPS
// and WIGB_CASES come from the command line.  Test infrastructure:
// tests/test_emu_cpu.py builds it and compares the result with the oracle.
//
//   batch_emu params W_in W_out obs_out n_prop grid
//
// params: count x 14 doubles per instance: n_x, n_p, v4, v2, v1, v0, gamma,
// d_theta, d_lambda, dt, x_amplitude, p_amplitude, damping_f (0: |p|, 1:
// p^2 / sqrt(p^2 + f_eps)), f_eps; hbar = mass = 1.  W_in / W_out: the
// instances' (n_p, n_x) states one after another, complex64.  obs_out: count x
// (n_prop + 1) x 11 doubles.  grid: CTAs of every launch.
#include "shim.h"
#include "wig_jit_batch.cuh"

#include <algorithm>
#include <map>

namespace {

// the host's FP32 twiddle: among the float pairs within 2 ulp of exp(-2 pi i m / n), the
// one with |w|^2 closest to 1 (ties: the closest in angle)
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

// wigb_create's per-instance float tables: [r_lambda / n_x][masks / n_p][(cos, -sin) of the
// row-pair kinetic ratio] and [r_theta][sign(p) f(p)][theta / n_p]
void instance_tables(wig::BInst& b, std::vector<float>* ft) {
  const int nx = b.n_x, np = b.n_p;
  b.ft_x = (int)ft->size();
  for (int k = 0; k < nx; ++k) {
    const double lam = b.dlambda * (((k + nx / 2) % nx) - 0.5 * nx);
    ft->push_back((float)(exp(-b.D_lambda * lam * lam) / (double)nx));
  }
  const double x_max = b.dx * (nx - 1.) / 2.;
  for (int k = 0; k < nx; ++k) {
    const double x = b.dx * (((k + nx / 2) % nx) - 0.5 * nx);
    const double w2 = (10. * b.dx) * (10. * b.dx);
    const double m1 = 1. - exp(-(x - x_max) * (x - x_max) / w2), m2 = 1. - exp(-(x + x_max) * (x + x_max) / w2);
    ft->push_back((float)(m1 * m2 / (double)np));
  }
  for (int k = 0; k < nx; ++k) {
    const int lj = k < nx / 2 ? k : k - nx;
    double t = b.dt * b.dp * b.dlambda * (double)lj / (b.mass * 2. * M_PI);
    t -= rint(t);
    ft->push_back((float)cos(2. * M_PI * t));
    ft->push_back((float)(-sin(2. * M_PI * t)));
  }
  b.ft_p = (int)ft->size();
  for (int k = 0; k < np; ++k) {
    const double th = b.dtheta * (((k + np / 2) % np) - 0.5 * np);
    ft->push_back((float)exp(-b.D_theta * th * th * b.dt));
  }
  for (int k = 0; k < np; ++k) {
    const double p = b.dp * (((k + np / 2) % np) - 0.5 * np);
    const double f = b.ff == 0 ? fabs(p) : p * p / sqrt(p * p + b.f_eps);
    ft->push_back((float)(p >= 0. ? f : -f));
  }
  for (int k = 0; k < np; ++k) {
    const double th = b.dtheta * (((k + np / 2) % np) - 0.5 * np);
    ft->push_back((float)(th / (double)np));
  }
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
  if (argc != 7) {
    std::fprintf(stderr, "usage: %s params W_in W_out obs_out n_prop grid\n", argv[0]);
    return 2;
  }
  const long n_prop = std::atol(argv[5]);
  const int grid = std::atoi(argv[6]);
  FILE* pf = std::fopen(argv[1], "rb");
  if (!pf) return 4;
  std::vector<double> prm;
  double v;
  while (std::fread(&v, sizeof v, 1, pf) == 1) prm.push_back(v);
  std::fclose(pf);
  constexpr int NPRM = 14;
  const int count = (int)(prm.size() / NPRM);
  if (count < 1 || n_prop < 1 || grid < 1) return 2;

  // wigb_create
  std::vector<wig::BInst> inst(count);
  std::vector<int> cls;
  for (int i = 0; i < count; ++i) {
    cls.push_back((int)prm[NPRM * i]);
    cls.push_back((int)prm[NPRM * i + 1]);
  }
  std::sort(cls.begin(), cls.end());
  cls.erase(std::unique(cls.begin(), cls.end()), cls.end());
  std::vector<float2> tw;
  std::map<int, int> tw_off;
  for (int n : cls) {
    tw_off[n] = (int)tw.size();
    rf_twiddles(n, &tw);
  }
  std::vector<float> ft;
  long long off = 0;
  for (int i = 0; i < count; ++i) {
    const double* q = &prm[NPRM * i];
    wig::BInst& b = inst[i];
    std::memset(&b, 0, sizeof(b));
    const int nx = (int)q[0], np = (int)q[1];
    const double gamma = q[6], xa = q[10], pa = q[11];
    b.n_x = nx; b.n_p = np;
    b.damp = gamma != 0. ? 1 : 0;
    b.ff = (int)q[12];
    b.f_eps = q[13];
    b.off = off;
    off += (long long)nx * np;
    b.tw_x = tw_off[nx]; b.tw_p = tw_off[np];
    b.dt = q[9]; b.hbar = 1.; b.mass = 1.;
    b.dx = 2. * xa / nx; b.dp = 2. * pa / np;
    b.dtheta = 2. * M_PI / (2. * pa); b.dlambda = 2. * M_PI / (2. * xa);
    b.D_theta = q[7]; b.D_lambda = q[8];
    b.v4 = q[2]; b.v2 = q[3]; b.v1 = q[4]; b.v0 = q[5];
    const double g = b.dt * gamma, c1 = 2. / 3. * g, c2 = g, c3 = 2. * g;
    b.cl_k1 = (c1 + c2) != 0. ? c1 * c2 / (c1 + c2) : 0.;
    b.cl_k12 = c1 + c2;
    b.cl_c3 = c3;
    instance_tables(b, &ft);
  }
  // wigb_set_warps: work lists, instances ordered by decreasing per-item cost
  std::vector<int> order(count);
  for (int i = 0; i < count; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
    return (long long)inst[a].n_p * (inst[a].damp ? 4 : 1) > (long long)inst[b].n_p * (inst[b].damp ? 4 : 1);
  });
  std::vector<int2> xi, pi;
  for (int i : order) {
    wig::BInst& b = inst[i];
    const int rpb = wig::bx_rows(b.n_x, WIGB_WARPS), cpb = wig::bp_cols(b.n_p, WIGB_WARPS);
    if (b.n_p % rpb || b.n_x % cpb) return 2;
    b.xitem0 = (int)xi.size();
    b.n_xitems = b.n_p / rpb;
    for (int r = 0; r < b.n_p; r += rpb) xi.push_back(make_int2(i, r));
    b.pitem0 = (int)pi.size();
    b.n_pitems = b.n_x / cpb;
    for (int c = 0; c < b.n_x; c += cpb) pi.push_back(make_int2(i, c));
  }
  std::vector<float2> W((size_t)off);
  if (!read_all(argv[2], W.data(), W.size())) return 4;
  std::vector<double> partials(pi.size() * wig::NACC, 0.);
  std::vector<unsigned> counters(count, 0u), tickets(2, 0u);
  std::vector<double2> scale(count, make_double2(1., 0.));
  std::vector<double> obs((size_t)count * (n_prop + 1) * wig::NOBS, 0.);

  wig::BArgs A{};
  A.inst = inst.data(); A.xitems = xi.data(); A.pitems = pi.data();
  A.W = W.data(); A.tw = tw.data(); A.ft = ft.data(); A.partials = partials.data();
  A.counters = counters.data(); A.tickets = tickets.data(); A.scale = scale.data();
  A.obs = obs.data(); A.obs_stride = (int)(n_prop + 1);
  const int nxi = (int)xi.size(), npi = (int)pi.size();

  // wigb_launch_run: reduce (normalisation, sample 0), then per step x-pass and p-pass, then scale
  emu_launch(grid, WIGB_NT, [&] { wigb_reduce(A, npi, 1, 0); });
  for (long n = 0; n < n_prop; ++n) {
    emu_launch(grid, WIGB_NT, [&] { wigb_xpass(A, nxi); });
    const int sample = (int)(n + 1);
    emu_launch(grid, WIGB_NT, [&] { wigb_ppass(A, npi, sample); });
  }
  emu_launch(grid, WIGB_NT, [&] { wigb_scale(A, npi); });
  if (tickets[0] != 0u || tickets[1] != 0u) {
    std::fprintf(stderr, "work-list tickets not reset: %u %u\n", tickets[0], tickets[1]);
    return 5;
  }
  if (!write_all(argv[3], W.data(), W.size())) return 4;
  if (!write_all(argv[4], obs.data(), obs.size())) return 4;
  return 0;
}
