// Dirac3D: host side of the dirac3_* entry points (include/wigner_b200.h),
// GPU_Dirac3D (GPU_Dirac3D.py:616-1500).  The kernels (wig_dirac3.cuh,
// wig_jit_dirac3.cuh) are compiled by NVRTC per instance with the instance's
// potential strings and '%f' constants, as the reference's SourceModule calls do.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "../../include/wigner_b200.h"
#include "wig_dirac3.cuh"
#include "wig_host.h"
#include "wig_dirac3_src.inc"   // kJitDirac3Source (generated by build.py)

using namespace wighost;

namespace {

constexpr int kMaxCta = 148 * 16;   // grid-stride passes: at most 16 CTAs per SM

struct Dirac3Plan {
  int rows, xnt, yc, ynt, zc, znt, snt;
  // largest Stockham radix / CTAs per SM of each pass: radix 16 only where it fits the register
  // budget without spilling (the z-pass: 126 registers, 3.00 vs 3.08 ms per 256^3 step)
  int xr = 8, yr = 8, zr = 16, xmb = 3, ymb = 4, zmb = 2;
  int gx, gy, gz, gn;
  int smem_x, smem_y, smem_z;
  double dX, dY, dZ, dPx, dPy, dPz;
  std::string src;
};

bool pow2_16_512(int n) { return n >= 16 && n <= 512 && (n & (n - 1)) == 0; }

int d3_plan(const dirac3_desc* d, Dirac3Plan* P) {
  if (!d) return fail(WIG_ERR_ARG, "dirac3: null descriptor");
  if (d->abi_version != WIG_ABI_VERSION)
    return fail(WIG_ERR_ARG, "dirac3: abi_version %d != %d", d->abi_version, WIG_ABI_VERSION);
  if (!pow2_16_512(d->n_x) || !pow2_16_512(d->n_y) || !pow2_16_512(d->n_z))
    return fail(WIG_ERR_ARG, "dirac3: grid %d x %d x %d: each axis must be a power of two in [16, 512]", d->n_x,
                d->n_y, d->n_z);
  if (!(d->x_amplitude > 0) || !(d->y_amplitude > 0) || !(d->z_amplitude > 0))
    return fail(WIG_ERR_ARG, "dirac3: amplitudes must be > 0");
  if (!std::isfinite(d->dt) || !std::isfinite(d->c) || !(d->hbar > 0) || !std::isfinite(d->hbar))
    return fail(WIG_ERR_ARG, "dirac3: dt and c must be finite, hbar > 0");
  // the K mix divides by E = c sqrt(p^2 + (m c / 2)^2), zero at p = 0 when m = 0
  if (!(d->mass > 0) || !std::isfinite(d->mass)) return fail(WIG_ERR_ARG, "dirac3: mass must be > 0");
  if (d->constants != WIG_CONST_CUDA_F && d->constants != WIG_CONST_EXACT)
    return fail(WIG_ERR_ARG, "dirac3: unknown constants mode %d", d->constants);
  if (d->precision != WIG_PREC_C128) return fail(WIG_ERR_UNSUPPORTED, "dirac3: precision %d not available", d->precision);
  const std::string A0 = expr_or(d->a0, "0."), A1 = expr_or(d->a1, "0."), A2 = expr_or(d->a2, "0."),
                    A3 = expr_or(d->a3, "0.");
  if (!safe_expr(A0) || !safe_expr(A1) || !safe_expr(A2) || !safe_expr(A3))
    return fail(WIG_ERR_ARG, "dirac3: expression strings may not contain ; { } # quotes or unbalanced ()");
  const int NX = d->n_x, NY = d->n_y, NZ = d->n_z, cm = d->constants;
  P->rows = clampi(512 / NX, 1, NY * NZ);
  P->xnt = round_warp(clampi(4 * P->rows * NX / 8, 32, 256));
  P->yc = clampi(2048 / NY, 2, NX);
  P->ynt = round_warp(clampi(NY * P->yc / 8, 32, 256));
  P->zc = clampi(1024 / NZ, 1, NX);
  // WIG_D3_TILING="rows,yc,zc" overrides the tile shapes for tuning runs (powers of two, clamped)
  if (const char* t = getenv("WIG_D3_TILING")) {
    int v[3] = {0, 0, 0};
    if (sscanf(t, "%d,%d,%d", &v[0], &v[1], &v[2]) == 3) {
      auto p2 = [](int x) { return x > 0 && (x & (x - 1)) == 0; };
      if (p2(v[0])) P->rows = clampi(v[0], 1, NY * NZ);
      if (p2(v[1])) P->yc = clampi(v[1], 1, NX);
      if (p2(v[2])) P->zc = clampi(v[2], 1, NX);
      P->xnt = round_warp(clampi(4 * P->rows * NX / 8, 32, 256));
      P->ynt = round_warp(clampi(NY * P->yc / 8, 32, 256));
    }
  }
  P->znt = round_warp(clampi(4 * P->zc * NZ / 8, 32, 256));
  // WIG_D3_RADIX="xr,yr,zr,xmb,ymb,zmb" overrides the radix caps (8 or 16) and CTAs per SM for tuning runs
  if (const char* t = getenv("WIG_D3_RADIX")) {
    int v[6] = {0, 0, 0, 0, 0, 0};
    if (sscanf(t, "%d,%d,%d,%d,%d,%d", &v[0], &v[1], &v[2], &v[3], &v[4], &v[5]) == 6) {
      auto rad = [](int x, int d) { return (x == 8 || x == 16) ? x : d; };
      P->xr = rad(v[0], P->xr); P->yr = rad(v[1], P->yr); P->zr = rad(v[2], P->zr);
      if (v[3] > 0) P->xmb = clampi(v[3], 1, 8);
      if (v[4] > 0) P->ymb = clampi(v[4], 1, 8);
      if (v[5] > 0) P->zmb = clampi(v[5], 1, 8);
    }
  }
  P->snt = 256;
  P->gx = clampi(NY * NZ / P->rows, 1, kMaxCta);
  P->gy = clampi(4 * NZ * (NX / P->yc), 1, kMaxCta);
  P->gz = clampi(NY * (NX / P->zc), 1, kMaxCta);
  P->gn = clampi((int)((4L * NX * NY * NZ) / (4L * P->snt)), 1, 1184);
  P->smem_x = wig::padded_size(4 * P->rows * NX) * (int)sizeof(double2);
  P->smem_y = wig::padded_size(NY * P->yc) * (int)sizeof(double2);
  P->smem_z = wig::padded_size(4 * P->zc * NZ) * (int)sizeof(double2);
  // GPU_Dirac3D.py:637-683
  P->dX = 2. * d->x_amplitude / (double)NX;
  P->dY = 2. * d->y_amplitude / (double)NY;
  P->dZ = 2. * d->z_amplitude / (double)NZ;
  P->dPx = 2 * (M_PI / P->dX) / NX;
  P->dPy = 2 * (M_PI / P->dY) / NY;
  P->dPz = 2 * (M_PI / P->dZ) / NZ;
  // the names the reference's kernels define (:690-700), visible to the expressions
  struct { const char* name; double v; } consts[] = {
      {"hBar", d->hbar}, {"mass", d->mass}, {"c", d->c},     {"dt", d->dt},   {"dX", P->dX},
      {"dY", P->dY},     {"dZ", P->dZ},     {"dPx", P->dPx}, {"dPy", P->dPy}, {"dPz", P->dPz}};
  std::string src = kMathPrelude;
  for (auto& c : consts) src += "__constant__ double " + std::string(c.name) + "=" + fmt_const(c.v, cm) + ";";
  src += "\nstruct UserPhys {\n  double cf[8];\n";
  const std::string* As[4] = {&A0, &A1, &A2, &A3};
  for (int i = 0; i < 4; ++i)
    src += "  __device__ __forceinline__ double A" + std::to_string(i) +
           "(double t, double x, double y, double z) const { return (" + *As[i] + "); }\n";
  src += "};\n";
  char macros[768];
  snprintf(macros, sizeof(macros),
           "#define D3_NX %d\n#define D3_NY %d\n#define D3_NZ %d\n#define D3_ROWS %d\n#define D3_XNT %d\n"
           "#define D3_YC %d\n#define D3_YNT %d\n#define D3_ZC %d\n#define D3_ZNT %d\n#define D3_SNT %d\n"
           "#define D3_XR %d\n#define D3_YR %d\n#define D3_ZR %d\n#define D3_XMB %d\n#define D3_YMB %d\n"
           "#define D3_ZMB %d\n",
           NX, NY, NZ, P->rows, P->xnt, P->yc, P->ynt, P->zc, P->znt, P->snt, P->xr, P->yr, P->zr, P->xmb,
           P->ymb, P->zmb);
  src += macros;
  src += kJitDirac3Source;
  P->src.swap(src);
  return WIG_OK;
}

}  // namespace

struct dirac3_handle {
  int device = 0;
  dirac3_desc d{};
  wig::Dirac3Args a{};
  Dirac3Plan P;
  CUfunction f_x = nullptr, f_yf = nullptr, f_yi = nullptr, f_z = nullptr, f_n = nullptr, f_nf = nullptr;
  DevBuf bufs;
  double* obs = nullptr;
  size_t obs_cap = 0;
  double2* stage = nullptr;   // device copy used by dirac3_run_host
};

extern "C" int dirac3_jit_check(const dirac3_desc* d, char* log, int64_t log_cap) {
  Dirac3Plan P;
  if (int rc = d3_plan(d, &P)) { copy_log(g_last_error, log, log_cap); return rc; }
  std::vector<char> cubin;
  std::string lg;
  int rc = nvrtc_compile_locked(P.src, &cubin, &lg, true);
  copy_log(rc ? g_last_error : lg, log, log_cap);
  return rc;
}

extern "C" int dirac3_create(const dirac3_desc* d, dirac3_handle** out) {
  if (!out) return fail(WIG_ERR_ARG, "dirac3_create: null argument");
  *out = nullptr;
  dirac3_handle* h = new dirac3_handle();
  if (int rc = d3_plan(d, &h->P)) { delete h; return rc; }
  h->d = *d;
  cudaError_t e = cudaGetDevice(&h->device);
  if (e == cudaSuccess) e = cudaFree(0);
  if (e != cudaSuccess) {
    delete h;
    return fail(WIG_ERR_CUDA, "dirac3_create: %s", cudaGetErrorString(e));
  }
  const Dirac3Plan& P = h->P;
  CUmodule mod;
  int rc = get_module(P.src, h->device, &mod);
  if (!rc) rc = get_fn(mod, "d3_xpass", &h->f_x, P.smem_x);
  if (!rc) rc = get_fn(mod, "d3_ypass_fwd", &h->f_yf, P.smem_y);
  if (!rc) rc = get_fn(mod, "d3_ypass_inv", &h->f_yi, P.smem_y);
  if (!rc) rc = get_fn(mod, "d3_zpass", &h->f_z, P.smem_z);
  if (!rc) rc = get_fn(mod, "d3_norm", &h->f_n, 0);
  if (!rc) rc = get_fn(mod, "d3_norm_fin", &h->f_nf, 0);
  if (rc) { delete h; return rc; }

  const int cm = d->constants, NX = d->n_x, NY = d->n_y, NZ = d->n_z;
  wig::Dirac3Args& a = h->a;
  a.hbar = kval(d->hbar, cm); a.mass = kval(d->mass, cm); a.c = kval(d->c, cm); a.dt = kval(d->dt, cm);
  a.dX = kval(P.dX, cm); a.dY = kval(P.dY, cm); a.dZ = kval(P.dZ, cm);
  a.dPx = kval(P.dPx, cm); a.dPy = kval(P.dPy, cm); a.dPz = kval(P.dPz, cm);
  a.dX_e = P.dX; a.dY_e = P.dY; a.dZ_e = P.dZ; a.dPx_e = P.dPx; a.dPy_e = P.dPy; a.dPz_e = P.dPz;
  for (int i = 0; i < 8; ++i) a.coef[i] = d->coef[i];
  std::vector<double2> twx = twiddles(NX), twy = twiddles(NY), twz = twiddles(NZ);
  const size_t npart_x = (size_t)(P.gx * wig::D3X > P.gn ? P.gx * wig::D3X : P.gn);
  const double init[2] = {1.0, 0.0};   // scale, s1
  double2 *twx_d, *twy_d, *twz_d;
  double *px0, *px1, *pp, *sc;
  DevBuf& B = h->bufs;
  rc = B.alloc(&twx_d, NX, twx.data());
  if (!rc) rc = B.alloc(&twy_d, NY, twy.data());
  if (!rc) rc = B.alloc(&twz_d, NZ, twz.data());
  if (!rc) rc = B.alloc(&px0, npart_x);
  if (!rc) rc = B.alloc(&px1, npart_x);
  if (!rc) rc = B.alloc(&pp, (size_t)P.gz * wig::D3P);
  if (!rc) rc = B.alloc(&sc, 2, init);
  if (rc) { B.free_all(); delete h; return rc; }
  a.tw_x = twx_d; a.tw_y = twy_d; a.tw_z = twz_d;
  a.part_x[0] = px0; a.part_x[1] = px1; a.part_p = pp;
  a.scale = sc; a.s1 = sc + 1;
  a.n_x_cta = P.gx; a.n_z_cta = P.gz;
  *out = h;
  return WIG_OK;
}

extern "C" int dirac3_run(dirac3_handle* h, void* psi_dev, int64_t t_index0, int64_t n_steps, uint32_t flags,
                          double* obs_host, void* stream) {
  if (!h || !psi_dev) return fail(WIG_ERR_ARG, "dirac3_run: null handle or psi");
  if (((uintptr_t)psi_dev & 15) != 0) return fail(WIG_ERR_ARG, "dirac3_run: psi must be 16-byte aligned");
  if (n_steps < 1) return fail(WIG_ERR_ARG, "dirac3_run: n_steps must be >= 1");
  int cur;
  WIG_CUDA(cudaGetDevice(&cur));
  if (cur != h->device) return fail(WIG_ERR_ARG, "dirac3_run: current device %d != handle device %d", cur, h->device);
  if (int rc = ensure_obs(&h->obs, &h->obs_cap, (size_t)n_steps * wig::D3NOBS)) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  const Dirac3Plan& P = h->P;
  double2* psi = (double2*)psi_dev;
  const double dt = h->d.dt;
  int normalise = (flags & WIG_RUN_CONTINUE) ? 0 : 1;
  if (normalise) {   // Normalize_GPU before the loop (:1323)
    long n = 4L * h->d.n_x * h->d.n_y * h->d.n_z;
    void* nargs[] = {&h->a, &psi, &n};
    if (int rc = launch(h->f_n, P.gn, P.snt, 0, st, nargs)) return rc;
    int ncta = P.gn;
    void* fargs[] = {&h->a, &ncta};
    if (int rc = launch(h->f_nf, 1, P.snt, 0, st, fargs)) return rc;
  }
  {
    int mode = 0, parity = 0;
    double tA = 0., tobs = dt * (double)(t_index0 + 1);
    long long prev = 0;
    double* obs_prev = nullptr;
    void* args[] = {&h->a, &psi, &mode, &parity, &normalise, &tA, &tobs, &prev, &obs_prev};
    if (int rc = launch(h->f_x, P.gx, P.xnt, P.smem_x, st, args)) return rc;
  }
  for (int64_t k = 1; k <= n_steps; ++k) {
    void* cargs[] = {&h->a, &psi};
    if (int rc = launch(h->f_yf, P.gy, P.ynt, P.smem_y, st, cargs)) return rc;
    if (int rc = launch(h->f_z, P.gz, P.znt, P.smem_z, st, cargs)) return rc;
    if (int rc = launch(h->f_yi, P.gy, P.ynt, P.smem_y, st, cargs)) return rc;
    int mode = (k == n_steps) ? 2 : 1, parity = (int)(k & 1), nrm = 0;
    double tA = dt * (double)(t_index0 + k), tobs = dt * (double)(t_index0 + k + 1);
    long long prev = (long long)(t_index0 + k);
    double* obs_prev = h->obs + (size_t)(k - 1) * wig::D3NOBS;
    void* args[] = {&h->a, &psi, &mode, &parity, &nrm, &tA, &tobs, &prev, &obs_prev};
    if (int rc = launch(h->f_x, P.gx, P.xnt, P.smem_x, st, args)) return rc;
  }
  if (obs_host) {
    const size_t nobs = (size_t)n_steps * wig::D3NOBS;
    WIG_CUDA(cudaMemcpyAsync(obs_host, h->obs, nobs * sizeof(double), cudaMemcpyDeviceToHost, st));
    WIG_CUDA(cudaStreamSynchronize(st));
    return check_finite(obs_host, nobs, "dirac3_run observables");
  }
  return WIG_OK;
}

extern "C" int dirac3_run_host(dirac3_handle* h, const void* psi_in, void* psi_out, int64_t t_index0,
                               int64_t n_steps, uint32_t flags, double* obs_host, void* stream) {
  if (!h || !psi_in || !psi_out) return fail(WIG_ERR_ARG, "dirac3_run_host: null argument");
  const size_t bytes = 4 * (size_t)h->d.n_x * h->d.n_y * h->d.n_z * sizeof(double2);
  if (!h->stage) {
    void* p = nullptr;
    WIG_CUDA(cudaMalloc(&p, bytes));
    h->stage = (double2*)p;
  }
  cudaStream_t st = (cudaStream_t)stream;
  WIG_CUDA(cudaMemcpyAsync(h->stage, psi_in, bytes, cudaMemcpyHostToDevice, st));
  if (int rc = dirac3_run(h, h->stage, t_index0, n_steps, flags, obs_host, stream)) return rc;
  WIG_CUDA(cudaMemcpyAsync(psi_out, h->stage, bytes, cudaMemcpyDeviceToHost, st));
  WIG_CUDA(cudaStreamSynchronize(st));
  return WIG_OK;
}

extern "C" int dirac3_destroy(dirac3_handle* h) {
  if (!h) return WIG_OK;
  cudaDeviceSynchronize();
  h->bufs.free_all();
  if (h->obs) cudaFree(h->obs);
  if (h->stage) cudaFree(h->stage);
  delete h;
  return WIG_OK;
}
