// Adjoint (differentiable) FP32 Wigner2D form: host side of the wiga_* /
// wig_step_adjoint entry points (include/wigner_b200.h).  The kernels
// (wig_adjoint.cuh, wig_jit_adjoint.cuh) are compiled by NVRTC per grid size.
// No counterpart in the reference.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/wigner_b200.h"
#include "wig_adjoint.cuh"
#include "wig_host.h"
#include "wig_batch_host.h"   // register-FFT twiddle tables
#include "wig_adjoint_src.inc"   // kJitAdjointSource (generated by build.py)

using namespace wighost;

struct wiga_handle {
  int device = 0;
  wiga_desc d{};
  wig::AArgs a{};
  DevBuf bufs;
  CUfunction fx = nullptr, fp = nullptr, fpt = nullptr, ffin = nullptr;
  int pw = 1, grid_x = 1, grid_p = 1, smem_x = 0, smem_p = 0, smem_pt = 0;
  double* partials = nullptr;
};

namespace {

bool pow2_64_1024(int n) { return n >= 64 && n <= 1024 && (n & (n - 1)) == 0; }

int check_desc(const wiga_desc* d) {
  if (!d) return fail(WIG_ERR_ARG, "wiga: null descriptor");
  if (d->abi_version != WIG_ABI_VERSION)
    return fail(WIG_ERR_ARG, "wiga: abi_version %d, library %d", d->abi_version, WIG_ABI_VERSION);
  if (!pow2_64_1024(d->n_x) || !pow2_64_1024(d->n_p))
    return fail(WIG_ERR_ARG, "wiga: grid %d x %d, grids must be powers of two in [64, 1024]", d->n_x, d->n_p);
  if (!(d->x_amplitude > 0) || !(d->p_amplitude > 0) || !(d->hbar != 0) || !(d->mass != 0) ||
      !std::isfinite(d->dt))
    return fail(WIG_ERR_ARG, "wiga: amplitudes > 0, hbar and mass nonzero, dt finite");
  return WIG_OK;
}

// p-pass tile: 4 columns (32-byte row segments)
int p_warps(int n_p) { return 4 / wig::rf_spw(n_p) > 0 ? 4 / wig::rf_spw(n_p) : 1; }

std::string source(const wiga_desc* d) {
  char head[160];
  snprintf(head, sizeof(head), "#define WIGA_NX %d\n#define WIGA_NP %d\n#define WIGA_PW %d\n", d->n_x, d->n_p,
           p_warps(d->n_p));
  return std::string(head) + kJitAdjointSource;
}

}  // namespace

extern "C" int wiga_jit_check(const wiga_desc* d, char* log, int64_t log_cap) {
  if (int rc = check_desc(d)) {
    copy_log(g_last_error, log, log_cap);
    return rc;
  }
  std::vector<char> cubin;
  std::string lg;
  int rc = nvrtc_compile_locked(source(d), &cubin, &lg, true);
  copy_log(rc ? g_last_error : lg, log, log_cap);
  return rc;
}

extern "C" int wiga_destroy(wiga_handle* h) {
  if (!h) return WIG_OK;
  cudaDeviceSynchronize();
  h->bufs.free_all();
  delete h;
  return WIG_OK;
}

extern "C" int wiga_create(const wiga_desc* d, wiga_handle** out) {
  if (!out) return fail(WIG_ERR_ARG, "wiga_create: null output");
  *out = nullptr;
  if (int rc = check_desc(d)) return rc;
  int device = 0;
  WIG_CUDA(cudaGetDevice(&device));
  WIG_CUDA(cudaFree(0));
  wiga_handle* h = new wiga_handle();
  h->device = device;
  h->d = *d;
  const int nx = d->n_x, np = d->n_p;
  wig::AArgs& a = h->a;
  a.n_x = nx; a.n_p = np;
  a.dt = d->dt; a.hbar = d->hbar; a.mass = d->mass;
  a.dx = 2. * d->x_amplitude / nx; a.dp = 2. * d->p_amplitude / np;
  a.dtheta = 2. * M_PI / (2. * d->p_amplitude); a.dlambda = 2. * M_PI / (2. * d->x_amplitude);
  a.v4 = d->v4; a.v2 = d->v2; a.v0 = d->v0;
  std::vector<float2> twx, twp;
  rf_twiddles(nx, &twx);
  rf_twiddles(np, &twp);
  // per-frequency / per-column factors (expPLambda_source :153, expPotential_source :117-123), FP64 then rounded
  std::vector<float> rtab(nx), mm(nx), rth(np);
  const double x_max = a.dx * (nx - 1.) / 2., w2 = (10. * a.dx) * (10. * a.dx);
  for (int k = 0; k < nx; ++k) {
    const double j = ((k + nx / 2) % nx) - 0.5 * nx;
    const double lam = a.dlambda * j, x = a.dx * j;
    rtab[k] = (float)(exp(-d->d_lambda * lam * lam) / (double)nx);
    const double m1 = 1. - exp(-(x - x_max) * (x - x_max) / w2), m2 = 1. - exp(-(x + x_max) * (x + x_max) / w2);
    mm[k] = (float)(m1 * m2 / (double)np);
  }
  for (int k = 0; k < np; ++k) {
    const double th = a.dtheta * (((k + np / 2) % np) - 0.5 * np);
    rth[k] = (float)exp(-d->d_theta * th * th * d->dt);
  }
  float2 *twx_d, *twp_d;
  float *rtab_d, *mm_d, *rth_d;
  int rc = h->bufs.alloc(&twx_d, twx.size(), twx.data());
  if (!rc) rc = h->bufs.alloc(&twp_d, twp.size(), twp.data());
  if (!rc) rc = h->bufs.alloc(&rtab_d, rtab.size(), rtab.data());
  if (!rc) rc = h->bufs.alloc(&mm_d, mm.size(), mm.data());
  if (!rc) rc = h->bufs.alloc(&rth_d, rth.size(), rth.data());
  h->pw = p_warps(np);
  const int spw_x = wig::rf_spw(nx), spw_p = wig::rf_spw(np), ct = h->pw * spw_p;
  h->grid_x = np / spw_x;
  h->grid_p = nx / ct;
  h->smem_x = spw_x * (nx + (wig::rf_g(nx) == 8 ? 8 : 0)) * (int)sizeof(float2);
  h->smem_p = ct * np * (int)sizeof(float2);
  h->smem_pt = 2 * ct * np * (int)sizeof(float2);
  if (!rc) rc = h->bufs.alloc(&h->partials, (size_t)h->grid_p);
  if (rc) { wiga_destroy(h); return rc; }
  a.tw_x = twx_d; a.tw_p = twp_d; a.rtab = rtab_d; a.mm = mm_d; a.rth = rth_d;
  CUmodule mod;
  rc = get_module(source(d), device, &mod);
  if (!rc) rc = get_fn(mod, "wiga_xpass", &h->fx, h->smem_x);
  if (!rc) rc = get_fn(mod, "wiga_ppass", &h->fp, h->smem_p);
  if (!rc) rc = get_fn(mod, "wiga_ppass_T", &h->fpt, h->smem_pt);
  if (!rc) rc = get_fn(mod, "wiga_grad_finalize", &h->ffin, 0);
  if (rc) { wiga_destroy(h); return rc; }
  *out = h;
  return WIG_OK;
}

static int check_ptr(const void* p, const char* what) {
  if (!p) return fail(WIG_ERR_ARG, "%s: null pointer", what);
  if (((uintptr_t)p & 15) != 0) return fail(WIG_ERR_ARG, "%s: device buffers must be 16-byte aligned", what);
  return WIG_OK;
}

static int check_device(wiga_handle* h, const char* what) {
  int cur = -1;
  WIG_CUDA(cudaGetDevice(&cur));
  if (cur != h->device) return fail(WIG_ERR_ARG, "%s: current device %d != handle device %d", what, cur, h->device);
  return WIG_OK;
}

extern "C" int wiga_forward(wiga_handle* h, void* W_dev, const double* eps_dev, int64_t step0, int64_t n_steps,
                            void* Y_dev, void* stream) {
  if (!h) return fail(WIG_ERR_ARG, "wiga_forward: null handle");
  if (int rc = check_ptr(W_dev, "wiga_forward W")) return rc;
  if (int rc = check_ptr(eps_dev, "wiga_forward eps")) return rc;
  if (Y_dev)
    if (int rc = check_ptr(Y_dev, "wiga_forward Y")) return rc;
  if (step0 < 0 || n_steps < 0) return fail(WIG_ERR_ARG, "wiga_forward: step0 and n_steps must be >= 0");
  if (int rc = check_device(h, "wiga_forward")) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  const size_t plane = (size_t)h->d.n_x * h->d.n_p;
  float2* W = (float2*)W_dev;
  float sgn = 1.f;
  for (int64_t n = 0; n < n_steps; ++n) {
    float2* Y = Y_dev ? (float2*)Y_dev + (size_t)n * plane : W;
    const float2* Wc = W;
    void* xa[] = {&h->a, (void*)&Wc, &Y, &sgn};
    if (int rc = launch(h->fx, h->grid_x, 32, h->smem_x, st, xa)) return rc;
    const float2* Yc = Y;
    long long step = (long long)(step0 + n);
    void* pa[] = {&h->a, (void*)&Yc, &W, (void*)&eps_dev, &step};
    if (int rc = launch(h->fp, h->grid_p, h->pw * 32, h->smem_p, st, pa)) return rc;
  }
  return WIG_OK;
}

extern "C" int wig_step_adjoint(wiga_handle* h, void* lam_dev, const void* Y_dev, const double* eps_dev,
                                int64_t step, double* grad_dev, void* stream) {
  if (!h) return fail(WIG_ERR_ARG, "wig_step_adjoint: null handle");
  if (int rc = check_ptr(lam_dev, "wig_step_adjoint lam")) return rc;
  if (int rc = check_ptr(Y_dev, "wig_step_adjoint Y")) return rc;
  if (int rc = check_ptr(eps_dev, "wig_step_adjoint eps")) return rc;
  if (!grad_dev || ((uintptr_t)grad_dev & 7) != 0) return fail(WIG_ERR_ARG, "wig_step_adjoint: bad grad pointer");
  if (step < 0) return fail(WIG_ERR_ARG, "wig_step_adjoint: step must be >= 0");
  if (int rc = check_device(h, "wig_step_adjoint")) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  float2* lam = (float2*)lam_dev;
  const float2* Y = (const float2*)Y_dev;
  long long s = (long long)step;
  void* pa[] = {&h->a, &lam, (void*)&Y, (void*)&eps_dev, &s, &h->partials};
  if (int rc = launch(h->fpt, h->grid_p, h->pw * 32, h->smem_pt, st, pa)) return rc;
  int n = h->grid_p;
  void* fa[] = {&h->partials, &n, &grad_dev, &s};
  if (int rc = launch(h->ffin, 1, 32, 0, st, fa)) return rc;
  const float2* lc = lam;
  float sgn = -1.f;
  void* xa[] = {&h->a, (void*)&lc, &lam, &sgn};
  return launch(h->fx, h->grid_x, 32, h->smem_x, st, xa);
}
