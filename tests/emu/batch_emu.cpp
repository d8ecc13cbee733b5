// Host execution of the batched Wigner2D kernels (csrc/wig_jit_batch.cuh)
// in the launch sequence of wigb_run (csrc/wig_capi.cu: wigb_launch_run), over
// the tables wigb_create builds (csrc/wig_batch_host.h, shared with the
// library) and the work lists of wigb_set_warps.  WIGB_WARPS, WIGB_PREC and
// WIGB_CASES come from the command line.  Test infrastructure:
// tests/test_emu_cpu.py builds it and compares the result with the oracle.
//
//   batch_emu params W_in W_out obs_out n_prop grid
//
// params: count x 14 doubles per instance: n_x, n_p, v4, v2, v1, v0, gamma,
// d_theta, d_lambda, dt, x_amplitude, p_amplitude, damping_f (0: |p|, 1:
// p^2 / sqrt(p^2 + f_eps)), f_eps; hbar = mass = 1.  W_in / W_out: the
// instances' (n_p, n_x) real states one after another, float32.  obs_out:
// count x (n_prop + 1) x 11 doubles.  grid: CTAs of every launch.
#include "shim.h"
#include "wig_jit_batch.cuh"
#include "wig_batch_host.h"

#include <algorithm>
#include <map>

namespace {

// the fields of wigb_instance (include/wigner_b200.h) that batch_instance_setup reads
struct Inst {
  int n_x, n_p, damping_f;
  double x_amplitude, p_amplitude, hbar, mass, dt, d_theta, d_lambda, gamma, f_eps, v4, v2, v1, v0;
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
  std::vector<double2> tw64;
  std::map<int, int> tw_off;
  wighost::batch_twiddles(cls, &tw, &tw64, &tw_off);
  std::vector<float> ft;
  std::vector<double> fd;
  long long off = 0;
  for (int i = 0; i < count; ++i) {
    const double* q = &prm[NPRM * i];
    Inst d{};
    d.n_x = (int)q[0]; d.n_p = (int)q[1];
    d.v4 = q[2]; d.v2 = q[3]; d.v1 = q[4]; d.v0 = q[5];
    d.gamma = q[6]; d.d_theta = q[7]; d.d_lambda = q[8]; d.dt = q[9];
    d.x_amplitude = q[10]; d.p_amplitude = q[11];
    d.damping_f = (int)q[12]; d.f_eps = q[13];
    d.hbar = 1.; d.mass = 1.;
    wig::BInst& b = inst[i];
    std::memset(&b, 0, sizeof(b));
    wighost::batch_instance_setup(d, b, &ft, &fd);
    b.off = off;
    off += (long long)d.n_x * d.n_p;
    b.tw_x = tw_off[d.n_x]; b.tw_p = tw_off[d.n_p];
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
  std::vector<float> W((size_t)off);
  if (!read_all(argv[2], W.data(), W.size())) return 4;
  std::vector<double> partials(pi.size() * wig::NACC, 0.);
  std::vector<unsigned> counters(count, 0u), tickets(2, 0u);
  std::vector<double> scale(count, 1.);
  std::vector<double> obs((size_t)count * (n_prop + 1) * wig::NOBS, 0.);

  wig::BArgs A{};
  A.inst = inst.data(); A.xitems = xi.data(); A.pitems = pi.data();
  A.W = W.data(); A.tw = tw.data(); A.tw64 = tw64.data(); A.ft = ft.data(); A.fd = fd.data();
  A.partials = partials.data();
  unsigned status = 0;
  A.counters = counters.data(); A.tickets = tickets.data(); A.scale = scale.data(); A.status = &status;
  A.obs = obs.data(); A.obs_stride = (int)(n_prop + 1);
  const int nxi = (int)xi.size(), npi = (int)pi.size();

  // dynamic shared memory of the passes (wigb_compile: the largest size class)
  size_t smx = (size_t)wigb_xexch_max() * sizeof(float2) + (WIGB_XSTAGE ? (size_t)wigb_xstage_max() * sizeof(float) : 0),
         smp = 0;
  for (int n : cls) smp = std::max(smp, (size_t)wig::bp_smem(n, WIGB_WARPS) * sizeof(float2));
  // wigb_launch_run: reduce (normalisation, sample 0), then per step x-pass and p-pass, then scale
  emu_launch(grid, WIGB_NT, [&] { wigb_reduce(A, npi, 1, 0); });
  for (long n = 0; n < n_prop; ++n) {
    A.step = (unsigned)n;
    emu_launch(grid, WIGB_NT, [&] { wigb_xpass(A, nxi); }, smx);
    const int sample = (int)(n + 1);
    emu_launch(grid, WIGB_NT, [&] { wigb_ppass(A, npi, sample); }, smp);
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
