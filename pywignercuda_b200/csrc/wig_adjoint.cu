// Adjoint (differentiable) Wigner2D form: host side of the wiga_* /
// wig_step_adjoint entry points (include/wigner_b200.h).  The kernels
// (wig_adjoint.cuh, wig_jit_adjoint.cuh) are compiled by NVRTC per grid size
// and precision.  No counterpart in the reference.
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
#include "wig_batch_host.h"     // register-FFT twiddle tables
#include "wig_adjoint_host.h"
#include "wig_adjoint_src.inc"   // kJitAdjointSource (generated by build.py)

using namespace wighost;

struct wiga_handle {
  int device = 0;
  wiga_desc d{};
  wig::AArgs a{};
  DevBuf bufs;
  CUfunction fx = nullptr, fp = nullptr, fpt = nullptr, ffin = nullptr, ffwd = nullptr, fsc = nullptr,
             frs = nullptr, fdot = nullptr, fcoef = nullptr;
  int pw = 1, grid_x = 1, grid_p = 1, smem_x = 0, smem_p = 0, grid_d = 1;
  size_t esize = 8;                 // bytes per element of the state
  double* part = nullptr;           // CTA partials (max of 3 per p-pass CTA, 2 per dot CTA)
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
  if (d->precision != WIGA_PREC_C64 && d->precision != WIGA_PREC_C128)
    return fail(WIG_ERR_ARG, "wiga: precision must be WIGA_PREC_C64 or WIGA_PREC_C128");
  if (!std::isfinite(d->gamma) || !(d->f_eps >= 0.))
    return fail(WIG_ERR_ARG, "wiga: gamma must be finite and f_eps >= 0");
  return WIG_OK;
}

std::string source(const wiga_desc* d) {
  char head[200];
  snprintf(head, sizeof(head), "#define WIGA_NX %d\n#define WIGA_NP %d\n#define WIGA_PW %d\n#define WIGA_PREC %d\n",
           d->n_x, d->n_p, adjoint_p_warps(d->n_p), d->precision);
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
  const bool c128 = d->precision == WIGA_PREC_C128;
  h->esize = c128 ? 16 : 8;
  wig::AArgs& a = h->a;
  AdjTables t;
  adjoint_setup(*d, a, &t);
  int rc = WIG_OK;
  if (c128) {
    std::vector<double2> twx, twp;
    rf_twiddles64(nx, &twx);
    rf_twiddles64(np, &twp);
    double2 *x_d = nullptr, *p_d = nullptr;
    rc = h->bufs.alloc(&x_d, twx.size(), twx.data());
    if (!rc) rc = h->bufs.alloc(&p_d, twp.size(), twp.data());
    a.tw_x = x_d;
    a.tw_p = p_d;
  } else {
    std::vector<float2> twx, twp;
    rf_twiddles(nx, &twx);
    rf_twiddles(np, &twp);
    float2 *x_d = nullptr, *p_d = nullptr;
    rc = h->bufs.alloc(&x_d, twx.size(), twx.data());
    if (!rc) rc = h->bufs.alloc(&p_d, twp.size(), twp.data());
    a.tw_x = x_d;
    a.tw_p = p_d;
  }
  double *rtab_d = nullptr, *mm_d = nullptr, *rth_d = nullptr, *sfp_d = nullptr, *ths_d = nullptr;
  double2* sc_d = nullptr;
  const double2 sc_init[3] = {make_double2(1., 0.), make_double2(1., 0.), make_double2(0., 0.)};
  if (!rc) rc = h->bufs.alloc(&rtab_d, t.rtab.size(), t.rtab.data());
  if (!rc) rc = h->bufs.alloc(&mm_d, t.mm.size(), t.mm.data());
  if (!rc) rc = h->bufs.alloc(&rth_d, t.rth.size(), t.rth.data());
  if (!rc) rc = h->bufs.alloc(&sfp_d, t.sfp.size(), t.sfp.data());
  if (!rc) rc = h->bufs.alloc(&ths_d, t.ths.size(), t.ths.data());
  if (!rc) rc = h->bufs.alloc(&sc_d, (size_t)3, sc_init);   // pend, coef[2]
  h->pw = adjoint_p_warps(np);
  const int spw_x = wig::rf_spw(nx), spw_p = wig::rf_spw(np), ct = h->pw * spw_p;
  h->grid_x = np / spw_x;
  h->grid_p = nx / ct;
  h->grid_d = 148;
  h->smem_x = spw_x * (nx + (wig::rf_g(nx) == 8 ? 8 : 0)) * (int)h->esize;
  h->smem_p = 2 * ct * np * (int)h->esize;
  if (!rc) rc = h->bufs.alloc(&h->part, (size_t)3 * std::max(h->grid_p, h->grid_d));
  if (rc) { wiga_destroy(h); return rc; }
  a.rtab = rtab_d; a.mm = mm_d; a.rth = rth_d; a.sfp = sfp_d; a.ths = ths_d;
  a.pend = sc_d;
  a.coef = sc_d + 1;
  CUmodule mod;
  rc = get_module(source(d), device, &mod);
  if (!rc) rc = get_fn(mod, "wiga_xpass", &h->fx, h->smem_x);
  if (!rc) rc = get_fn(mod, "wiga_ppass", &h->fp, h->smem_p);
  if (!rc) rc = get_fn(mod, "wiga_ppass_T", &h->fpt, h->smem_p);
  if (!rc) rc = get_fn(mod, "wiga_grad_finalize", &h->ffin, 0);
  if (!rc) rc = get_fn(mod, "wiga_fwd_finalize", &h->ffwd, 0);
  if (!rc) rc = get_fn(mod, "wiga_scale", &h->fsc, 0);
  if (!rc) rc = get_fn(mod, "wiga_reset_pend", &h->frs, 0);
  if (!rc) rc = get_fn(mod, "wiga_dot", &h->fdot, 0);
  if (!rc) rc = get_fn(mod, "wiga_adj_coef", &h->fcoef, 0);
  if (rc) { wiga_destroy(h); return rc; }
  *out = h;
  return WIG_OK;
}

extern "C" int wiga_set_potential(wiga_handle* h, double v4, double v2, double v0) {
  if (!h) return fail(WIG_ERR_ARG, "wiga_set_potential: null handle");
  if (!std::isfinite(v4) || !std::isfinite(v2) || !std::isfinite(v0))
    return fail(WIG_ERR_ARG, "wiga_set_potential: coefficients must be finite");
  h->a.v4 = v4;
  h->a.v2 = v2;
  h->a.v0 = v0;
  h->d.v4 = v4;
  h->d.v2 = v2;
  h->d.v0 = v0;
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
                            void* Y_dev, void* U_dev, void* s_dev, void* stream) {
  if (!h) return fail(WIG_ERR_ARG, "wiga_forward: null handle");
  if (int rc = check_ptr(W_dev, "wiga_forward W")) return rc;
  if (int rc = check_ptr(eps_dev, "wiga_forward eps")) return rc;
  if (Y_dev)
    if (int rc = check_ptr(Y_dev, "wiga_forward Y")) return rc;
  if (U_dev)
    if (int rc = check_ptr(U_dev, "wiga_forward U")) return rc;
  if (s_dev)
    if (int rc = check_ptr(s_dev, "wiga_forward s")) return rc;
  if ((U_dev || s_dev) && !h->a.damped) return fail(WIG_ERR_ARG, "wiga_forward: U and s are records of damped steps");
  if (step0 < 0 || n_steps < 0) return fail(WIG_ERR_ARG, "wiga_forward: step0 and n_steps must be >= 0");
  if (int rc = check_device(h, "wiga_forward")) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  const size_t plane = (size_t)h->d.n_x * h->d.n_p;
  char* W = (char*)W_dev;
  double sgn = 1.;
  for (int64_t n = 0; n < n_steps; ++n) {
    char* Y = Y_dev ? (char*)Y_dev + (size_t)n * plane * h->esize : W;
    char* U = U_dev ? (char*)U_dev + (size_t)n * plane * h->esize : nullptr;
    const char* Wc = W;
    int use_pend = (h->a.damped && n > 0) ? 1 : 0;
    void* xa[] = {&h->a, (void*)&Wc, &Y, &sgn, &use_pend};
    if (int rc = launch(h->fx, h->grid_x, 32, h->smem_x, st, xa)) return rc;
    const char* Yc = Y;
    long long step = (long long)(step0 + n);
    void* pa[] = {&h->a, (void*)&Yc, &W, &U, (void*)&eps_dev, &step, &h->part};
    if (int rc = launch(h->fp, h->grid_p, h->pw * 32, h->smem_p, st, pa)) return rc;
    if (h->a.damped) {
      int np = h->grid_p;
      void* fa[] = {&h->a, &h->part, &np, &s_dev, &step};
      if (int rc = launch(h->ffwd, 1, 32, 0, st, fa)) return rc;
    }
  }
  if (h->a.damped && n_steps > 0) {
    long long n = (long long)plane;
    void* sa[] = {&h->a, &W, &n};
    if (int rc = launch(h->fsc, 148 * 4, 256, 0, st, sa)) return rc;
    void* ra[] = {&h->a};
    if (int rc = launch(h->frs, 1, 32, 0, st, ra)) return rc;
  }
  return WIG_OK;
}

namespace {

// The launches of adjoint step `step` (arguments checked by the caller).
int adjoint_step_launch(wiga_handle* h, char* lam, const void* Y_dev, const void* U_dev, const void* s_dev,
                        const double* eps_dev, long long s, double* grad_dev, cudaStream_t st) {
  if (h->a.damped) {
    long long n = (long long)h->d.n_x * h->d.n_p;
    const char* lc = lam;
    void* da[] = {(void*)&lc, (void*)&U_dev, &n, &h->part};
    if (int rc = launch(h->fdot, h->grid_d, 256, 0, st, da)) return rc;
    int nd = h->grid_d;
    void* ca[] = {&h->a, &h->part, &nd, (void*)&s_dev, &s};
    if (int rc = launch(h->fcoef, 1, 32, 0, st, ca)) return rc;
  }
  void* pa[] = {&h->a, &lam, (void*)&Y_dev, (void*)&eps_dev, &s, &h->part};
  if (int rc = launch(h->fpt, h->grid_p, h->pw * 32, h->smem_p, st, pa)) return rc;
  int n = h->grid_p;
  void* fa[] = {&h->part, &n, &grad_dev, &s};
  if (int rc = launch(h->ffin, 1, 32, 0, st, fa)) return rc;
  const char* lc = lam;
  double sgn = -1.;
  int use_pend = 0;
  void* xa[] = {&h->a, (void*)&lc, &lam, &sgn, &use_pend};
  return launch(h->fx, h->grid_x, 32, h->smem_x, st, xa);
}

int check_adjoint_args(wiga_handle* h, void* lam_dev, const void* Y_dev, const void* U_dev, const void* s_dev,
                       const double* eps_dev, int64_t step, double* grad_dev, const char* what) {
  if (!h) return fail(WIG_ERR_ARG, "%s: null handle", what);
  if (int rc = check_ptr(lam_dev, "adjoint lam")) return rc;
  if (int rc = check_ptr(Y_dev, "adjoint Y")) return rc;
  if (int rc = check_ptr(eps_dev, "adjoint eps")) return rc;
  if (h->a.damped) {
    if (int rc = check_ptr(U_dev, "adjoint U")) return rc;
    if (int rc = check_ptr(s_dev, "adjoint s")) return rc;
  }
  if (!grad_dev || ((uintptr_t)grad_dev & 7) != 0) return fail(WIG_ERR_ARG, "%s: bad grad pointer", what);
  if (step < 0) return fail(WIG_ERR_ARG, "%s: step must be >= 0", what);
  return check_device(h, what);
}

}  // namespace

extern "C" int wig_step_adjoint(wiga_handle* h, void* lam_dev, const void* Y_dev, const void* U_dev,
                                const void* s_dev, const double* eps_dev, int64_t step, double* grad_dev,
                                void* stream) {
  if (int rc = check_adjoint_args(h, lam_dev, Y_dev, U_dev, s_dev, eps_dev, step, grad_dev, "wig_step_adjoint"))
    return rc;
  return adjoint_step_launch(h, (char*)lam_dev, Y_dev, U_dev, s_dev, eps_dev, (long long)step, grad_dev,
                             (cudaStream_t)stream);
}

extern "C" int wiga_adjoint_sweep(wiga_handle* h, void* lam_dev, const void* Y_dev, const void* U_dev,
                                  const void* s_dev, const double* eps_dev, int64_t step0, int64_t n_steps,
                                  double* grad_dev, void* stream) {
  if (n_steps < 1) return fail(WIG_ERR_ARG, "wiga_adjoint_sweep: n_steps must be >= 1");
  if (int rc = check_adjoint_args(h, lam_dev, Y_dev, U_dev, s_dev, eps_dev, step0, grad_dev, "wiga_adjoint_sweep"))
    return rc;
  const size_t plane = (size_t)h->d.n_x * h->d.n_p * h->esize;
  cudaStream_t st = (cudaStream_t)stream;
  for (int64_t k = n_steps - 1; k >= 0; --k) {
    const char* Yk = (const char*)Y_dev + (size_t)k * plane;
    const char* Uk = U_dev ? (const char*)U_dev + (size_t)k * plane : nullptr;
    if (int rc = adjoint_step_launch(h, (char*)lam_dev, Yk, Uk, s_dev, eps_dev, (long long)(step0 + k), grad_dev, st))
      return rc;
  }
  return WIG_OK;
}
