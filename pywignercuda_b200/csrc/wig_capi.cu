// C ABI of the B200 Wigner2D / Dirac2D propagators (see include/wigner_b200.h).
//
// Host side: descriptor validation, the instance's kernel constants (the
// reference's '%f' formatting, GPU_Wigner2D_FFT.py:833-842 /
// GPU_Dirac2D.py:358-367), NVRTC compilation of the fused kernels with the
// user's expression strings pasted in (the reference's SourceModule calls,
// GPU_Wigner2D_FFT.py:869-906 / GPU_Dirac2D.py:369-388), per-instance tables,
// and the launch sequence of the hot loop (GPU_Wigner2D_FFT.Run :1843-1914,
// GPU_Dirac2D.Run :1055-1111).
//
// The library links the CUDA runtime statically and reaches the driver API
// and NVRTC only at run time (cudaGetDriverEntryPointByVersion, dlopen), so it
// loads on machines without a GPU driver.
#include <cuda_runtime.h>
#include <cudaTypedefs.h>
#include <nvrtc.h>
#include <dlfcn.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/wigner_b200.h"
#include "wig_dirac.cuh"
#include "wig_batch.cuh"
#include "wig_batch_host.h"
#include "wig_wigner_rf.cuh"
#include "wig_device_src.inc"   // kJitWignerSource, kJitDiracSource (generated by build.py)
#include "wig_host.h"

namespace wighost {

// ------------------------------------------------------------------ errors
thread_local std::string g_last_error;

int fail(int code, const char* fmt, ...) {
  char buf[2048];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}


// ------------------------------------------------------------------ driver API
struct Driver {
  PFN_cuModuleLoadData load = nullptr;
  PFN_cuModuleGetFunction getf = nullptr;
  PFN_cuLaunchKernel launch = nullptr;
  PFN_cuFuncSetAttribute setattr = nullptr;
  PFN_cuGetErrorString errstr = nullptr;
  PFN_cuTensorMapEncodeTiled encode = nullptr;   // optional: TMA tile loads need it
  bool ok = false;
};

std::mutex g_mu;
Driver g_drv;

template <class F>
bool entry(const char* name, F& fn) {
  cudaDriverEntryPointQueryResult q;
  void* p = nullptr;
  if (cudaGetDriverEntryPointByVersion(name, &p, 12000, cudaEnableDefault, &q) != cudaSuccess ||
      q != cudaDriverEntryPointSuccess || !p)
    return false;
  fn = reinterpret_cast<F>(p);
  return true;
}

int driver(Driver** out) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_drv.ok) {
    if (!(entry("cuModuleLoadData", g_drv.load) && entry("cuModuleGetFunction", g_drv.getf) &&
          entry("cuLaunchKernel", g_drv.launch) && entry("cuFuncSetAttribute", g_drv.setattr) &&
          entry("cuGetErrorString", g_drv.errstr)))
      return fail(WIG_ERR_CUDA, "CUDA driver entry points unavailable (no GPU driver?)");
    if (!entry("cuTensorMapEncodeTiled", g_drv.encode)) g_drv.encode = nullptr;
    g_drv.ok = true;
  }
  *out = &g_drv;
  return WIG_OK;
}

const char* cu_err(CUresult r) {
  const char* s = nullptr;
  if (g_drv.errstr) g_drv.errstr(r, &s);
  return s ? s : "unknown CUDA driver error";
}

// ------------------------------------------------------------------ NVRTC
struct Nvrtc {
  decltype(&nvrtcCreateProgram) create = nullptr;
  decltype(&nvrtcCompileProgram) compile = nullptr;
  decltype(&nvrtcGetProgramLogSize) logsize = nullptr;
  decltype(&nvrtcGetProgramLog) log = nullptr;
  decltype(&nvrtcGetCUBINSize) cubinsize = nullptr;
  decltype(&nvrtcGetCUBIN) cubin = nullptr;
  decltype(&nvrtcDestroyProgram) destroy = nullptr;
  bool ok = false;
};
Nvrtc g_nvrtc;

int nvrtc(Nvrtc** out) {
  // caller holds g_mu
  if (!g_nvrtc.ok) {
    const char* names[] = {"libnvrtc.so.12", "/usr/local/cuda/lib64/libnvrtc.so.12", "libnvrtc.so"};
    void* h = nullptr;
    for (const char* n : names)
      if ((h = dlopen(n, RTLD_NOW | RTLD_LOCAL))) break;
    if (!h) return fail(WIG_ERR_NVRTC, "cannot load libnvrtc.so.12: %s", dlerror());
#define WIG_SYM(f, s)                                                                    \
  g_nvrtc.f = reinterpret_cast<decltype(g_nvrtc.f)>(dlsym(h, s));                        \
  if (!g_nvrtc.f) return fail(WIG_ERR_NVRTC, "libnvrtc: missing symbol %s", s);
    WIG_SYM(create, "nvrtcCreateProgram")
    WIG_SYM(compile, "nvrtcCompileProgram")
    WIG_SYM(logsize, "nvrtcGetProgramLogSize")
    WIG_SYM(log, "nvrtcGetProgramLog")
    WIG_SYM(cubinsize, "nvrtcGetCUBINSize")
    WIG_SYM(cubin, "nvrtcGetCUBIN")
    WIG_SYM(destroy, "nvrtcDestroyProgram")
#undef WIG_SYM
    g_nvrtc.ok = true;
  }
  *out = &g_nvrtc;
  return WIG_OK;
}

// Compiled modules, keyed by (device, source); kept for the process lifetime.
std::map<std::string, CUmodule> g_modules;

// NVRTC: source -> sm_100a CUBIN (no GPU needed).  Caller holds g_mu.
int nvrtc_compile(const std::string& src, std::vector<char>* cubin, std::string* log, bool verbose) {
  Nvrtc* nv;
  if (int rc = nvrtc(&nv)) return rc;
  nvrtcProgram prog;
  if (nv->create(&prog, src.c_str(), "wig_jit.cu", 0, nullptr, nullptr) != NVRTC_SUCCESS)
    return fail(WIG_ERR_NVRTC, "nvrtcCreateProgram failed");
  std::vector<const char*> opts = {"--gpu-architecture=sm_100a", "-std=c++17", "-lineinfo"};
  if (verbose) opts.push_back("--ptxas-options=-v");
  nvrtcResult cr = nv->compile(prog, (int)opts.size(), opts.data());
  size_t ls = 0;
  nv->logsize(prog, &ls);
  log->assign(ls, '\0');
  if (ls) nv->log(prog, &(*log)[0]);
  if (cr != NVRTC_SUCCESS) {
    nv->destroy(&prog);
    return fail(WIG_ERR_NVRTC, "expression strings failed to compile:\n%s", log->c_str());
  }
  size_t n = 0;
  nv->cubinsize(prog, &n);
  cubin->resize(n);
  nv->cubin(prog, cubin->data());
  nv->destroy(&prog);
  return WIG_OK;
}

bool env_verbose() {
  const char* v = getenv("WIG_JIT_VERBOSE");
  return v && *v && *v != '0';
}

int get_module(const std::string& src, int device, CUmodule* mod) {
  Driver* drv;
  if (int rc = driver(&drv)) return rc;
  std::lock_guard<std::mutex> lk(g_mu);
  const std::string key = std::to_string(device) + "\n" + src;
  auto it = g_modules.find(key);
  if (it != g_modules.end()) { *mod = it->second; return WIG_OK; }
  std::vector<char> cubin;
  std::string log;
  const bool verbose = env_verbose();
  if (int rc = nvrtc_compile(src, &cubin, &log, verbose)) return rc;
  if (verbose) fprintf(stderr, "[wigner_b200 jit]\n%s\n", log.c_str());
  CUresult r = drv->load(mod, cubin.data());
  if (r != CUDA_SUCCESS) return fail(WIG_ERR_CUDA, "cuModuleLoadData: %s", cu_err(r));
  g_modules[key] = *mod;
  return WIG_OK;
}

int copy_log(const std::string& log, char* out, int64_t cap) {
  if (out && cap > 0) {
    const size_t n = std::min((size_t)(cap - 1), log.size());
    memcpy(out, log.data(), n);
    out[n] = '\0';
  }
  return WIG_OK;
}

int get_fn(CUmodule mod, const char* name, CUfunction* f, int dyn_smem) {
  CUresult r = g_drv.getf(f, mod, name);
  if (r != CUDA_SUCCESS) return fail(WIG_ERR_CUDA, "cuModuleGetFunction(%s): %s", name, cu_err(r));
  // always raise the dynamic ceiling to the request: static shared memory counts against the
  // default 48 KB too, so a request just at 48 KB already needs the attribute
  if (dyn_smem > 0) {
    r = g_drv.setattr(*f, CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, dyn_smem);
    if (r != CUDA_SUCCESS) return fail(WIG_ERR_CUDA, "cuFuncSetAttribute(%s): %s", name, cu_err(r));
  }
  return WIG_OK;
}

int launch(CUfunction f, unsigned grid, unsigned block, unsigned smem, cudaStream_t st, void** args) {
  CUresult r = g_drv.launch(f, grid, 1, 1, block, 1, 1, smem, (CUstream)st, args, nullptr);
  if (r != CUDA_SUCCESS) return fail(WIG_ERR_CUDA, "cuLaunchKernel: %s", cu_err(r));
  return WIG_OK;
}

int launch2d(CUfunction f, unsigned gx, unsigned gy, unsigned block, unsigned smem, cudaStream_t st, void** args) {
  CUresult r = g_drv.launch(f, gx, gy, 1, block, 1, 1, smem, (CUstream)st, args, nullptr);
  if (r != CUDA_SUCCESS) return fail(WIG_ERR_CUDA, "cuLaunchKernel: %s", cu_err(r));
  return WIG_OK;
}

// ------------------------------------------------------------------ helpers
bool pow2_in_range(int n) { return n >= 16 && n <= 4096 && (n & (n - 1)) == 0; }
int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
int round_warp(int v) { return ((v + 31) / 32) * 32; }

// '%f' formatting of the reference (or exact), and the value the kernel sees.
std::string fmt_const(double v, int mode) {
  char b[64];
  snprintf(b, sizeof(b), mode == WIG_CONST_EXACT ? "%.17g" : "%f", v);
  return b;
}
double kval(double v, int mode) { return strtod(fmt_const(v, mode).c_str(), nullptr); }

// numpy linspace(-a, a - 2a/n, n) put through fftshift (GPU_Wigner2D_FFT.py:568-581)
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

// tw[m] = exp(-2 pi i m / n), extended precision, exact zeros on the axes
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

std::string expr_or(const char* s, const char* dflt) {
  if (!s) return dflt;
  std::string e(s);
  if (e.find_first_not_of(" \t\r\n") == std::string::npos) return dflt;
  return e;
}

bool safe_expr(const std::string& e) {
  // the expression is pasted between parentheses inside a function body: refuse
  // text that could close it or start a preprocessor directive
  int depth = 0;
  for (char ch : e) {
    if (ch == '(') ++depth;
    else if (ch == ')') { if (--depth < 0) return false; }
    else if (ch == ';' || ch == '{' || ch == '}' || ch == '#' || ch == '"' || ch == '\\') return false;
  }
  return depth == 0;
}

const char* kMathPrelude =
    "#ifndef M_PI\n#define M_PI 3.14159265358979323846\n#endif\n"
    "#ifndef M_E\n#define M_E 2.7182818284590452354\n#endif\n";

int nvrtc_compile_locked(const std::string& src, std::vector<char>* cubin, std::string* log, bool verbose) {
  std::lock_guard<std::mutex> lk(g_mu);
  return nvrtc_compile(src, cubin, log, verbose);
}

int occupancy(CUfunction f, int threads, int dyn_smem) {
  static PFN_cuOccupancyMaxActiveBlocksPerMultiprocessor occ = nullptr;
  if (!occ) entry("cuOccupancyMaxActiveBlocksPerMultiprocessor", occ);
  int n = 1;
  if (!occ || occ(&n, f, threads, dyn_smem) != CUDA_SUCCESS) n = 1;
  return n < 1 ? 1 : n;
}

int ensure_obs(double** buf, size_t* cap, size_t need) {
  if (need <= *cap) return WIG_OK;
  if (*buf) cudaFree(*buf);
  *buf = nullptr;
  *cap = 0;
  WIG_CUDA(cudaMalloc((void**)buf, need * sizeof(double)));
  *cap = need;
  return WIG_OK;
}

int check_finite(const double* v, size_t n, const char* what) {
  for (size_t i = 0; i < n; ++i)
    if (!std::isfinite(v[i])) return fail(WIG_ERR_NONFINITE, "%s: non-finite value at index %zu", what, i);
  return WIG_OK;
}

}  // namespace wighost

using namespace wighost;

// ======================================================================== Wigner
struct wig_handle {
  int device = 0;
  wig_desc d{};
  wig::WigArgs a{};
  CUfunction f_x = nullptr, f_p = nullptr, f_r = nullptr, f_fin = nullptr, f_scale = nullptr;
  CUfunction f_ox = nullptr, f_op = nullptr;   // ODM passes
  // Strang / Gross-Pitaevskii (GPU_Wigner2D_GPitaevskii)
  int strang = 0, gp = 0, smem_ph = 0, smem_gph = 0, n_chunks = 0;
  CUfunction f_ph = nullptr, f_phf = nullptr, f_gcs = nullptr, f_gm = nullptr, f_gph = nullptr;
  // Bloch (imaginary time)
  CUfunction f_bph = nullptr, f_bx = nullptr, f_gb = nullptr, f_br = nullptr, f_rs = nullptr, f_ba = nullptr;
  double* bloch_part = nullptr;                // [n_cta_r][wig::NBL]
  double2* rowsums = nullptr;                  // [n_p]
  double* bloch_psq = nullptr;                 // [1]
  double2* gp_chunks = nullptr;                // [n_p/16][n_x] column sums
  double* gp_P = nullptr;                      // [n_x] marginal
  double* gp_phase = nullptr;                  // [n_p][n_x]
  double* psq = nullptr;                       // per-step sum_x P^2 dx of the last run
  size_t psq_cap = 0;
  int64_t psq_n = 0;
  cudaStream_t last_stream = nullptr;
  int odm = 0, smem_odm_x = 0, smem_odm_p = 0;
  double2* odm_T = nullptr;                    // 5 planes of ODM intermediates
  double odm_coef[2] = {0., 0.}, odm_sign[2] = {1., -1.};
  int rf = 0;                                   // register-FFT x- and p-pass (wig_wigner_rf.cuh)
  int tma = 0, rf_c = 1;                        // the p-pass tile (rf_c columns) arrives by 2-D tensor copies
  wig::TensorMap tmap{};                        // tensor map of the W it was last encoded for
  const void* tmap_W = nullptr;
  int* status = nullptr;                        // [1] bounded-wait status of the kernels
  int xrows = 1, xnt = 256, pc = 1, pnt = 256, rnt = 256;
  int n_cta_x = 1, n_cta_p = 1, n_cta_r = 1;
  int smem_x = 0, smem_p = 0;
  DevBuf bufs;
  double* obs = nullptr;
  size_t obs_cap = 0;
  double2* scale = nullptr;
  double2* W_host_stage = nullptr;   // device copy used by wig_run_host
  std::vector<cudaEvent_t> ev;       // WIG_RUN_PROFILE: 3 events per step
  size_t ev_used = 0;
};

// Validation, tiling and the JIT source of one Wigner instance (no CUDA calls).
struct WigPlan {
  int rf = 0, rfxw = 4, rfpw = 2;   // register-FFT passes (wig_wigner_rf.cuh) and their warps per CTA
  int tma = 0;                      // their p-pass tile by 2-D tensor copies (WIG_TMA)
  int xrows, xnt, pc, pnt, rnt, n_cta_x, n_cta_p, n_cta_r, smem_x, smem_p, damp;
  int strang, gp, smem_ph, smem_gph;
  int xminb, pminb, xr, pr;
  int odm, smem_odm_x, smem_odm_p;
  double dX, dP, dTheta, dLambda;
  std::string src;
};

static int wig_plan(const wig_desc* d, WigPlan* P) {
  if (!d) return fail(WIG_ERR_ARG, "wig: null descriptor");
  if (d->abi_version != WIG_ABI_VERSION)
    return fail(WIG_ERR_ARG, "wig: abi_version %d != %d", d->abi_version, WIG_ABI_VERSION);
  if (!pow2_in_range(d->n_x) || !pow2_in_range(d->n_p))
    return fail(WIG_ERR_ARG, "grid %d x %d: n_x and n_p must be powers of two in [16, 4096]", d->n_x,
                d->n_p);
  if (!(d->x_amplitude > 0) || !(d->p_amplitude > 0) || !(d->hbar != 0) || !(d->mass != 0) ||
      !std::isfinite(d->dt))
    return fail(WIG_ERR_ARG, "amplitudes must be > 0, hbar and mass nonzero, dt finite");
  if (d->constants != WIG_CONST_CUDA_F && d->constants != WIG_CONST_EXACT)
    return fail(WIG_ERR_ARG, "unknown constants mode %d", d->constants);
  if (d->precision != WIG_PREC_C128) return fail(WIG_ERR_UNSUPPORTED, "precision %d not available", d->precision);
  const bool damped = d->gamma != 0.;
  if (damped && d->damping == WIG_DAMP_ODM && (d->n_lindblad < 1 || d->n_lindblad > 2))
    return fail(WIG_ERR_ARG, "n_lindblad must be 1 or 2");
  if (damped && d->damping == WIG_DAMP_ODM && !(d->l_material > 0))
    return fail(WIG_ERR_ARG, "ODM needs l_material > 0");
  if (d->potential_phase != WIG_PHASE_MOYAL && d->potential_phase != WIG_PHASE_KVN)
    return fail(WIG_ERR_ARG, "unknown potential_phase %d", d->potential_phase);
  if (d->potential_phase == WIG_PHASE_KVN && damped && d->damping == WIG_DAMP_ODM)
    return fail(WIG_ERR_UNSUPPORTED, "the KvN (Fokker-Planck) potential factor takes no ODM damping");
  if (d->splitting != WIG_SPLIT_LIE && d->splitting != WIG_SPLIT_STRANG_GP)
    return fail(WIG_ERR_ARG, "unknown splitting %d", d->splitting);
  if (d->splitting == WIG_SPLIT_STRANG_GP && d->potential_phase != WIG_PHASE_MOYAL)
    return fail(WIG_ERR_UNSUPPORTED, "Strang splitting takes the Moyal potential factor only");
  if (d->splitting != WIG_SPLIT_STRANG_GP && d->gp_coefficient != 0.)
    return fail(WIG_ERR_ARG, "gp_coefficient needs WIG_SPLIT_STRANG_GP");
  if (!std::isfinite(d->gp_coefficient)) return fail(WIG_ERR_ARG, "gp_coefficient must be finite");
  const std::string V = expr_or(d->potential, "0."), K = expr_or(d->kinetic, "0.5*p*p"),
                    F = expr_or(d->fp_damping, "fabs(p)"), DV = expr_or(d->dpotential, "0.");
  if (!safe_expr(V) || !safe_expr(K) || !safe_expr(F) || !safe_expr(DV))
    return fail(WIG_ERR_ARG, "expression strings may not contain ; { } # quotes or unbalanced ()");
  const int NX = d->n_x, NP = d->n_p, cm = d->constants;
  P->damp = (damped && d->damping == WIG_DAMP_CALDEIRA_LEGGETT) ? 1 : 0;
  P->odm = (damped && d->damping == WIG_DAMP_ODM) ? 1 : 0;

  // ---- tiling (defaults; WIG_TILING="xrows,xnt,xminb,pc,pnt,pminb" overrides for tuning runs)
  P->xrows = clampi(2048 / NX, 1, NP);
  P->xnt = round_warp(clampi(P->xrows * NX / 8, 32, 256));
  P->xminb = 3;
  // beyond 2048-point rows a thread holds two radix-8 butterflies per stage: 3 CTAs per SM
  // (80 registers) would spill ~1.4 KB per thread, 2 (128) spill a few bytes
  if ((P->xrows * NX / 8 + P->xnt - 1) / P->xnt > 1) P->xminb = 2;
  if (NX == 1024 && d->splitting == WIG_SPLIT_LIE) {
    // one 1024-point row per CTA of 128 threads, 8 CTAs per SM (64 registers, no spill): the
    // rows of a 1024^2 grid fill one wave (2.446 -> 2.293 ms per 16-replica Caldeira-Leggett step)
    P->xrows = 1;
    P->xnt = 128;
    P->xminb = 8;
  }
  P->pc = clampi(2048 / NP, 1, NX);
  P->pnt = round_warp(clampi(P->pc * NP / 8, 32, 256));
  P->pminb = P->damp ? 2 : 3;
  if ((P->pc * NP / 8 + P->pnt - 1) / P->pnt > 1) P->pminb = 2;   // as for the x-pass, beyond 2048 points
  if (const char* tv = getenv("WIG_TILING")) {
    int v[6];
    if (sscanf(tv, "%d,%d,%d,%d,%d,%d", &v[0], &v[1], &v[2], &v[3], &v[4], &v[5]) == 6) {
      if (v[0] > 0) P->xrows = clampi(v[0], 1, NP);
      if (v[1] > 0) P->xnt = round_warp(clampi(v[1], 32, 1024));
      if (v[2] > 0) P->xminb = v[2];
      if (v[3] > 0) P->pc = clampi(v[3], 1, NX);
      if (v[4] > 0) P->pnt = round_warp(clampi(v[4], 32, 1024));
      if (v[5] > 0) P->pminb = v[5];
    }
  }
  // WIG_RADIX="xr,pr": largest Stockham radix (8 or 16) of the x-pass / p-pass transforms, for tuning runs
  P->xr = 8;
  P->pr = 8;
  if (const char* tv = getenv("WIG_RADIX")) {
    int v[2];
    if (sscanf(tv, "%d,%d", &v[0], &v[1]) == 2) {
      if (v[0] == 8 || v[0] == 16) P->xr = v[0];
      if (v[1] == 8 || v[1] == 16) P->pr = v[1];
    }
  }
  P->rnt = 256;
  P->n_cta_x = NP / P->xrows;
  P->n_cta_p = NX / P->pc;
  P->n_cta_r = clampi(NX * NP / (4 * P->rnt), 1, 296);
  // shared layouts carry one padding slot per 8 elements (wig::padded_size)
  const int tile_x = wig::padded_size(P->xrows * NX) * (int)sizeof(double2);
  const int tile_p = wig::padded_size(P->pc * NP) * (int)sizeof(double2);
  P->smem_x = tile_x;
  P->smem_p = P->damp ? 2 * tile_p + 2 * NP * (int)sizeof(double) : tile_p;
  P->smem_odm_x = 2 * tile_x;
  P->smem_odm_p = 2 * tile_p;
  P->strang = d->splitting == WIG_SPLIT_STRANG_GP ? 1 : 0;
  P->gp = (P->strang && d->gp_coefficient != 0.) ? 1 : 0;
  P->smem_ph = tile_p;                                                     // first half: no damping
  P->smem_gph = (wig::padded_size(NX) + wig::padded_size(P->xrows * NX)) * (int)sizeof(double2);

  // ---- register-FFT passes (wig_wigner_rf.cuh) for Lie plans without ODM damping on
  // 64..1024-point axes, with the p-pass tile loaded by 2-D tensor copies: opt-in (WIG_RF="1",
  // or WIG_RF="xw,pw" with the warps per x-pass / p-pass CTA).  On the 1024^2 Caldeira-Leggett
  // case they measured slower than the Stockham passes (2.47 vs 2.18 ms per 16-replica step:
  // 255 registers a thread leave 5 warps per SM), so the Stockham passes are the default.
  const auto rf_size = [](int n) { return n >= 64 && n <= 1024; };
  P->rf = 0;
  if (const char* rv = getenv("WIG_RF")) {
    const int eligible = (!P->strang && !P->odm && rf_size(NX) && rf_size(NP)) ? 1 : 0;
    int v[2];
    if (sscanf(rv, "%d,%d", &v[0], &v[1]) == 2) {
      if (v[0] == 1 || v[0] == 2 || v[0] == 4 || v[0] == 8) P->rfxw = v[0];
      if (v[1] == 1 || v[1] == 2 || v[1] == 4 || v[1] == 8) P->rfpw = v[1];
      P->rf = eligible;
    } else if (atoi(rv) != 0) {
      P->rf = eligible;
    }
  }
  if (P->rf) {
    const int spx = wig::rf_spw(NX), spp = wig::rf_spw(NP);
    P->rfxw = std::min(P->rfxw, std::max(1, NP / spx));   // a CTA's rows within the grid
    P->rfpw = std::min(P->rfpw, std::max(1, NX / spp));
    while (P->rfpw > 1 && P->rfpw * spp > 8) P->rfpw /= 2;  // a tile of at most 8 columns (128-byte rows)
    // TMA tile loads: on unless WIG_TMA="0" (the thread loads fill the same layout)
    const char* tv = getenv("WIG_TMA");
    P->tma = (tv && atoi(tv) == 0) ? 0 : 1;
    P->xnt = 32 * P->rfxw;
    P->n_cta_x = NP / (P->rfxw * spx);
    P->smem_x = P->rfxw * spx * (NX + (wig::rf_g(NX) == 8 ? 8 : 0)) * (int)sizeof(double2);
    P->pnt = 32 * P->rfpw;
    P->n_cta_p = NX / (P->rfpw * spp);
    P->smem_p = (P->damp ? 2 : 1) * P->rfpw * spp * NP * (int)sizeof(double2) + 1024;   // + alignment slack
  }

  // ---- JIT source
  P->dX = 2. * d->x_amplitude / (double)NX;
  P->dP = 2. * d->p_amplitude / (double)NP;
  P->dTheta = 2. * M_PI / (2. * d->p_amplitude);
  P->dLambda = 2. * M_PI / (2. * d->x_amplitude);
  struct { const char* name; double v; } consts[] = {
      {"dt", d->dt}, {"dx", P->dX}, {"dp", P->dP}, {"dtheta", P->dTheta}, {"dlambda", P->dLambda},
      {"mass", d->mass}, {"hBar", d->hbar}, {"D_Theta", d->d_theta}, {"D_Lambda", d->d_lambda}};
  std::string src = kMathPrelude;
  for (auto& c : consts) src += "__constant__ double " + std::string(c.name) + "=" + fmt_const(c.v, cm) + ";";
  src += "\nstruct UserPhys {\n  double cf[8];\n";
  src += "  __device__ __forceinline__ double Potential(double t, double x) const { return (" + V + "); }\n";
  src += "  __device__ __forceinline__ double KineticEnergy(double p) const { return (" + K + "); }\n";
  src += "  __device__ __forceinline__ double f(double p) const { return (" + F + "); }\n";
  src += "  __device__ __forceinline__ double DPotential(double t, double x) const { return (" + DV + "); }\n};\n";
  char macros[512];
  snprintf(macros, sizeof(macros),
           "#define WIG_NX %d\n#define WIG_NP %d\n#define WIG_XROWS %d\n#define WIG_XNT %d\n"
           "#define WIG_KIN_STRING %d\n#define WIG_PC %d\n#define WIG_PNT %d\n"
           "#define WIG_DAMP %d\n#define WIG_RNT %d\n#define WIG_XMINB %d\n#define WIG_PMINB %d\n"
           "#define WIG_KVN %d\n#define WIG_STRANG %d\n#define WIG_XR %d\n#define WIG_PR %d\n",
           NX, NP, P->xrows, P->xnt, d->kinetic_from_string ? 1 : 0, P->pc, P->pnt, P->damp, P->rnt,
           P->xminb, P->pminb, d->potential_phase == WIG_PHASE_KVN ? 1 : 0, P->strang, P->xr, P->pr);
  src += macros;
  if (P->rf) {
    // 255 registers a thread (a 32-element FP64 sequence per lane is 128 of them)
    snprintf(macros, sizeof(macros),
             "#define WIG_RF 1\n#define WIG_RFXW %d\n#define WIG_RFPW %d\n#define WIG_RFXMB %d\n#define WIG_RFPMB %d\n",
             P->rfxw, P->rfpw, std::max(1, 8 / P->rfxw), std::max(1, 8 / P->rfpw));
    src += macros;
    if (P->tma) src += "#define WIG_TMA 1\n";
  }
  src += kJitWignerSource;
  P->src.swap(src);
  return WIG_OK;
}

extern "C" int wig_jit_check(const wig_desc* d, char* log, int64_t log_cap) {
  WigPlan P;
  if (int rc = wig_plan(d, &P)) { copy_log(g_last_error, log, log_cap); return rc; }
  std::lock_guard<std::mutex> lk(g_mu);
  std::vector<char> cubin;
  std::string lg;
  int rc = nvrtc_compile(P.src, &cubin, &lg, true);
  copy_log(rc ? g_last_error : lg, log, log_cap);
  return rc;
}

extern "C" int wig_create(const wig_desc* d, wig_handle** out) {
  if (!out) return fail(WIG_ERR_ARG, "wig_create: null argument");
  *out = nullptr;
  WigPlan P;
  if (int rc = wig_plan(d, &P)) return rc;
  int device = 0;
  WIG_CUDA(cudaGetDevice(&device));
  WIG_CUDA(cudaFree(0));
  wig_handle* h = new wig_handle();
  h->d = *d;
  h->device = device;
  const int NX = d->n_x, NP = d->n_p, cm = d->constants;
  h->xrows = P.xrows; h->xnt = P.xnt; h->pc = P.pc; h->pnt = P.pnt; h->rnt = P.rnt;
  h->n_cta_x = P.n_cta_x; h->n_cta_p = P.n_cta_p; h->n_cta_r = P.n_cta_r;
  h->smem_x = P.smem_x; h->smem_p = P.smem_p;
  h->odm = P.odm; h->smem_odm_x = P.smem_odm_x; h->smem_odm_p = P.smem_odm_p;
  const double dX = P.dX, dP = P.dP, dTheta = P.dTheta, dLambda = P.dLambda;
  const std::string& src = P.src;
  CUmodule mod;
  int rc = get_module(src, h->device, &mod);
  h->rf = P.rf;
  h->tma = P.tma;
  if (P.rf) h->rf_c = P.rfpw * wig::rf_spw(NP);
  if (h->tma && !g_drv.encode) { delete h; return fail(WIG_ERR_CUDA, "cuTensorMapEncodeTiled unavailable (set WIG_TMA=0)"); }
  if (!rc) rc = get_fn(mod, P.rf ? "wig_xpass_rf" : "wig_xpass", &h->f_x, h->smem_x);
  if (!rc) rc = get_fn(mod, P.rf ? "wig_ppass_rf" : "wig_ppass", &h->f_p, h->smem_p);
  if (!rc) rc = get_fn(mod, "wig_reduce", &h->f_r, 0);
  if (!rc) rc = get_fn(mod, "wig_finalize", &h->f_fin, 0);
  if (!rc) rc = get_fn(mod, "wig_scale", &h->f_scale, 0);
  CUfunction f_setup = nullptr;
  if (!rc) rc = get_fn(mod, "wig_setup", &f_setup, 0);
  if (!rc && h->odm) rc = get_fn(mod, "wig_odm_xpass", &h->f_ox, h->smem_odm_x);
  if (!rc && h->odm) rc = get_fn(mod, "wig_odm_ppass", &h->f_op, h->smem_odm_p);
  h->strang = P.strang; h->gp = P.gp; h->smem_ph = P.smem_ph; h->smem_gph = P.smem_gph;
  h->n_chunks = NP / 16;
  if (!rc && h->strang) rc = get_fn(mod, "wig_ppass_half", &h->f_ph, h->smem_ph);
  if (!rc && h->strang) rc = get_fn(mod, "wig_ppass_half_final", &h->f_phf, h->smem_p);
  if (!rc && h->gp) rc = get_fn(mod, "wig_gp_colsum", &h->f_gcs, 0);
  if (!rc && h->gp) rc = get_fn(mod, "wig_gp_marginal", &h->f_gm, 0);
  if (!rc && h->gp) rc = get_fn(mod, "wig_gp_phase", &h->f_gph, h->smem_gph);
  if (!rc && h->strang) rc = get_fn(mod, "wig_bloch_ppass", &h->f_bph, h->smem_ph);
  if (!rc && h->strang) rc = get_fn(mod, "wig_bloch_xpass", &h->f_bx, h->smem_x);
  if (!rc && h->strang) rc = get_fn(mod, "wig_bloch_reduce", &h->f_br, 0);
  if (!rc && h->strang) rc = get_fn(mod, "wig_rowsum", &h->f_rs, 0);
  if (!rc && h->strang) rc = get_fn(mod, "wig_bloch_axpy", &h->f_ba, 0);
  if (!rc && h->gp) rc = get_fn(mod, "wig_gp_bloch", &h->f_gb, h->smem_gph);
  if (rc) { delete h; return rc; }

  // ---- kernel arguments and tables
  wig::WigArgs& a = h->a;
  a.dt = kval(d->dt, cm); a.dx = kval(dX, cm); a.dp = kval(dP, cm);
  a.dtheta = kval(dTheta, cm); a.dlambda = kval(dLambda, cm); a.mass = kval(d->mass, cm);
  a.hbar = kval(d->hbar, cm); a.D_theta = kval(d->d_theta, cm); a.D_lambda = kval(d->d_lambda, cm);
  a.dX = dX; a.dP = dP; a.mass_exact = d->mass;
  {
    // CaldeiraDissipatorOrder3 (:1145-1157) coefficients c1 = 2/3 i dt gamma,
    // c2 = i dt gamma, c3 = 2 i dt gamma; Horner: k1 = c1 c2/(c1 + c2), k12 = c1 + c2
    const double g = d->dt * d->gamma;
    const double c1 = 2. / 3. * g, c2 = 2. / 2. * g, c3 = 2. * g;   // imaginary parts
    // c1 c2 / (c1 + c2) with c1 = i u, c2 = i v:  (i u)(i v)/(i (u+v)) = i u v/(u+v)
    const double k1 = (c1 + c2) != 0. ? c1 * c2 / (c1 + c2) : 0.;
    a.cl_k1 = make_double2(0., k1);
    a.cl_k12 = make_double2(0., c1 + c2);
    a.cl_c3 = make_double2(0., c3);
  }
  std::vector<double> xt = d->x_table ? std::vector<double>(d->x_table, d->x_table + NX) : shifted_range(d->x_amplitude, NX);
  std::vector<double> pt = d->p_table ? std::vector<double>(d->p_table, d->p_table + NP) : shifted_range(d->p_amplitude, NP);
  std::vector<double> tht = d->theta_table ? std::vector<double>(d->theta_table, d->theta_table + NP)
                                           : shifted_range(dTheta * NP / 2., NP);
  std::vector<double> ths(NP);
  for (int i = 0; i < NP; ++i) ths[i] = tht[i] * (1.0 / (double)NP);
  std::vector<double> dv(NX, 0.), v0(NX, 0.);
  if (d->dv_table) dv.assign(d->dv_table, d->dv_table + NX);
  if (d->v0_table) v0.assign(d->v0_table, d->v0_table + NX);
  std::vector<double2> twx = twiddles(NX), twp = twiddles(NP);
  double *x_d, *p_d, *dv_d, *v0_d, *ths_d, *rl_d, *rt_d, *m1_d, *m2_d, *sfp_d, *part_d;
  double2 *twx_d, *twp_d;
  const int nparts = std::max(std::max(h->n_cta_x, h->n_cta_p), h->n_cta_r);
  DevBuf& B = h->bufs;
  rc = B.alloc(&x_d, NX, xt.data());
  if (!rc) rc = B.alloc(&p_d, NP, pt.data());
  if (!rc) rc = B.alloc(&dv_d, NX, dv.data());
  if (!rc) rc = B.alloc(&v0_d, NX, v0.data());
  if (!rc) rc = B.alloc(&ths_d, NP, ths.data());
  if (!rc) rc = B.alloc(&rl_d, NX);
  if (!rc) rc = B.alloc(&rt_d, NP);
  if (!rc) rc = B.alloc(&m1_d, NX);
  if (!rc) rc = B.alloc(&m2_d, NX);
  if (!rc) rc = B.alloc(&sfp_d, NP);
  if (!rc) rc = B.alloc(&twx_d, NX, twx.data());
  if (!rc) rc = B.alloc(&twp_d, NP, twp.data());
  if (!rc) rc = B.alloc(&part_d, (size_t)nparts * wig::NACC);
  if (!rc) rc = B.alloc(&h->scale, 1);
  std::vector<double> lt = d->lambda_table ? std::vector<double>(d->lambda_table, d->lambda_table + NX)
                                           : shifted_range(dLambda * NX / 2., NX);
  double* lam_d = nullptr;
  if (!rc) rc = B.alloc(&lam_d, NX, lt.data());
  if (!rc && h->odm) rc = B.alloc(&h->odm_T, 5 * (size_t)NX * NP);
  // ODM steps do not keep sum W real: the samples need the imaginary moment sums too
  double* part_im_d = nullptr;
  if (!rc && h->odm) rc = B.alloc(&part_im_d, (size_t)nparts * wig::NIM);
  double* rth_d = nullptr;
  if (!rc) rc = B.alloc(&rth_d, NP);
  if (!rc && h->gp) rc = B.alloc(&h->gp_chunks, (size_t)h->n_chunks * NX);
  if (!rc && h->gp) rc = B.alloc(&h->gp_P, NX);
  if (!rc && h->gp) rc = B.alloc(&h->gp_phase, (size_t)NX * NP);
  if (!rc && h->strang) rc = B.alloc(&h->bloch_part, (size_t)h->n_cta_r * wig::NBL);
  if (!rc && h->strang) rc = B.alloc(&h->rowsums, (size_t)NP);
  if (!rc && h->gp) rc = B.alloc(&h->bloch_psq, (size_t)1);
  double2 *rtwx_d = nullptr, *rtwp_d = nullptr;
  if (!rc && h->rf) {
    std::vector<double2> rx, rp;
    rf_twiddles64(NX, &rx);
    rf_twiddles64(NP, &rp);
    rc = B.alloc(&rtwx_d, rx.size(), rx.data());
    if (!rc) rc = B.alloc(&rtwp_d, rp.size(), rp.data());
  }
  if (rc) { B.free_all(); delete h; return rc; }
  a.rtw_x = rtwx_d;
  a.rtw_p = rtwp_d;
  {
    int zero = 0;
    if (int rc2 = B.alloc(&h->status, (size_t)1, &zero)) { B.free_all(); delete h; return rc2; }
    a.status = h->status;
  }
  a.r_theta_half = rth_d;
  a.gp_coef = kval(d->gp_coefficient, cm);
  a.lambda_tab = lam_d;
  a.hbar_exact = d->hbar;
  a.L_material = d->l_material;
  for (int i = 0; i < 8; ++i) a.coef[i] = d->coef[i];
  // _Lindbladian_ODM scale dt*2*gamma*weight/n (n = 1, Order1), with 1/n_p folded in
  h->odm_coef[0] = d->dt * 2 * d->gamma * d->weight1 / 1. * (1.0 / (double)NP);
  h->odm_coef[1] = d->dt * 2 * d->gamma * d->weight2 / 1. * (1.0 / (double)NP);
  a.x_tab = x_d; a.p_tab = p_d; a.dV_tab = dv_d; a.V0_tab = v0_d; a.theta_s = ths_d;
  a.r_lambda = rl_d; a.r_theta = rt_d; a.mask1 = m1_d; a.mask2s = m2_d; a.sfp = sfp_d;
  a.tw_x = twx_d; a.tw_p = twp_d; a.partials = part_d; a.partials_im = part_im_d; a.n_partials = 0;
  {
    void* args[] = {&a, &rl_d, &rt_d, &m1_d, &m2_d, &sfp_d, &rth_d};
    rc = launch(f_setup, 8, 256, 0, 0, args);
    if (!rc) {
      cudaError_t e = cudaDeviceSynchronize();
      if (e != cudaSuccess) rc = fail(WIG_ERR_CUDA, "wig_setup: %s", cudaGetErrorString(e));
    }
    if (rc) { B.free_all(); delete h; return rc; }
  }
  *out = h;
  return WIG_OK;
}

// ---- one run, split so that several instances can be stepped in lock-step
struct WigRunState {
  wig::WigArgs a;
  double2* W;
  int64_t t_index0, n_prop;
  uint32_t flags;
  bool damped;
};

static int wig_run_check(wig_handle* h, void* W_dev, int64_t n_prop) {
  if (!h || !W_dev) return fail(WIG_ERR_ARG, "wig_run: null handle or W");
  if (((uintptr_t)W_dev & 15) != 0) return fail(WIG_ERR_ARG, "wig_run: W must be 16-byte aligned");
  if (n_prop < 0) return fail(WIG_ERR_ARG, "wig_run: n_prop < 0");
  int cur;
  WIG_CUDA(cudaGetDevice(&cur));
  if (cur != h->device) return fail(WIG_ERR_ARG, "wig_run: current device %d != handle device %d", cur, h->device);
  if (int rc = ensure_obs(&h->obs, &h->obs_cap, (size_t)(n_prop + 1) * WIG_NOBS)) return rc;
  if (h->gp)
    if (int rc = ensure_obs(&h->psq, &h->psq_cap, (size_t)std::max<int64_t>(n_prop, 1))) return rc;
  return WIG_OK;
}

static int wig_profile_prepare(wig_handle* h, int64_t n_prop) {
  const size_t need = 3 * (size_t)n_prop;
  while (h->ev.size() < need) {
    cudaEvent_t e;
    WIG_CUDA(cudaEventCreate(&e));
    h->ev.push_back(e);
  }
  h->ev_used = need;
  return WIG_OK;
}

static int wig_run_begin(wig_handle* h, WigRunState* S, void* W_dev, int64_t t_index0, int64_t n_prop,
                         uint32_t flags, cudaStream_t st) {
  S->a = h->a;
  S->W = (double2*)W_dev;
  S->t_index0 = t_index0;
  S->n_prop = n_prop;
  S->flags = flags;
  S->damped = h->d.gamma != 0. && !h->d.skip_normalise;   // whether damped steps renormalise
  if (flags & WIG_RUN_PROFILE) {
    if (int rc = wig_profile_prepare(h, n_prop)) return rc;
  } else {
    h->ev_used = 0;
  }
  void* args[] = {&S->a, &S->W};
  if (int rc = launch(h->f_r, h->n_cta_r, h->rnt, 0, st, args)) return rc;
  S->a.n_partials = h->n_cta_r;
  return WIG_OK;
}

// Gross-Pitaevskii phase of the current W into h->gp_phase: column sums, the
// marginal (with the pending normalisation of scale_mode; psq_out may be null)
// and the per-row phase.
static int wig_gp_terms(wig_handle* h, WigRunState* S, int scale_mode, double* psq_out, cudaStream_t st) {
  const int NX = h->d.n_x, NP = h->d.n_p, cnt = NX < 256 ? NX : 256;
  void* cargs[] = {&S->W, &h->gp_chunks};   // grid: columns x row chunks of 16
  if (int rc = launch2d(h->f_gcs, (unsigned)(NX / cnt), (unsigned)(NP / 16), (unsigned)cnt, 0, st, cargs)) return rc;
  int nch = h->n_chunks;
  void* margs[] = {&S->a, &h->gp_chunks, &nch, &scale_mode, &h->gp_P, &psq_out};
  if (int rc = launch(h->f_gm, 1, 256, 0, st, margs)) return rc;
  void* pargs[] = {&S->a, &h->gp_P, &h->gp_phase};
  return launch(h->f_gph, h->n_cta_x, h->xnt, h->smem_gph, st, pargs);
}

// One step of GPU_Wigner2D_GPitaevskii.Run (:1897-1975): [GP terms] half
// potential -> kinetic -> [GP terms] half potential -> damping.  The first
// half consumes the previous partials (sample n, normalisation on load).
static int wig_run_step_strang(wig_handle* h, WigRunState* S, int64_t n, cudaStream_t st) {
  const int first = (S->flags & WIG_RUN_CONTINUE) ? 0 : 1;
  int mode = (n == 0) ? first : (S->damped ? 2 : 0);
  double* obs_row = h->obs + (size_t)n * WIG_NOBS;
  const bool prof = h->ev_used != 0;
  double t = (double)(S->t_index0 + n) * h->d.dt;
  double* gph = h->gp ? h->gp_phase : nullptr;
  if (prof) WIG_CUDA(cudaEventRecord(h->ev[3 * n], st));
  if (h->gp)
    if (int rc = wig_gp_terms(h, S, mode, nullptr, st)) return rc;
  void* hargs[] = {&S->a, &S->W, &t, &mode, &obs_row, &gph};
  if (int rc = launch(h->f_ph, h->n_cta_p, h->pnt, h->smem_ph, st, hargs)) return rc;
  int zero = 0;
  double* none = nullptr;
  void* xargs[] = {&S->a, &S->W, &zero, &none};
  if (int rc = launch(h->f_x, h->n_cta_x, h->xnt, h->smem_x, st, xargs)) return rc;
  if (prof) WIG_CUDA(cudaEventRecord(h->ev[3 * n + 1], st));
  if (h->gp)
    if (int rc = wig_gp_terms(h, S, 0, h->psq + n, st)) return rc;
  void* fargs[] = {&S->a, &S->W, &t, &gph};
  if (int rc = launch(h->f_phf, h->n_cta_p, h->pnt, h->smem_p, st, fargs)) return rc;
  if (h->odm) {
    // Lindbladian_ODM_Order1 with weight 1, sign 1 (GPU_Wigner2D_GPitaevskii.Run :1966-1969)
    void* oxargs[] = {&S->a, &S->W, &h->odm_T};
    if (int rc = launch(h->f_ox, h->n_cta_x, h->xnt, h->smem_odm_x, st, oxargs)) return rc;
    double coef = h->odm_coef[0], sign = 1.;
    void* opargs[] = {&S->a, &S->W, &h->odm_T, &coef, &sign};
    if (int rc = launch(h->f_op, h->n_cta_p, h->pnt, h->smem_odm_p, st, opargs)) return rc;
  }
  if (prof) WIG_CUDA(cudaEventRecord(h->ev[3 * n + 2], st));
  S->a.n_partials = h->n_cta_p;
  return WIG_OK;
}

// The tensor map of the p-pass tile over W: (NP, NX) complex128 as a 2-D FP64 array of
// 2 NX x NP, boxes of 2 rf_c doubles x min(NP, 256) rows, the swizzle of a rf_c * 16-byte
// row (wig_wigner_rf.cuh: tma_sw).  The map holds W's address: it is encoded again for
// another W.
static int encode_tile_map(wig_handle* h, const void* W) {
  const int NX = h->d.n_x, NP = h->d.n_p, C = h->rf_c;
  CUtensorMap m;
  cuuint64_t dims[2] = {(cuuint64_t)2 * NX, (cuuint64_t)NP};
  cuuint64_t strides[1] = {(cuuint64_t)2 * NX * sizeof(double)};
  cuuint32_t box[2] = {(cuuint32_t)(2 * C), (cuuint32_t)(NP < 256 ? NP : 256)};
  cuuint32_t estr[2] = {1, 1};
  const CUtensorMapSwizzle swz = C == 1 ? CU_TENSOR_MAP_SWIZZLE_NONE
                                 : (C == 2 ? CU_TENSOR_MAP_SWIZZLE_32B
                                           : (C == 4 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_128B));
  CUresult r = g_drv.encode(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<void*>(W), dims, strides, box, estr,
                            CU_TENSOR_MAP_INTERLEAVE_NONE, swz, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(WIG_ERR_CUDA, "cuTensorMapEncodeTiled: %s", cu_err(r));
  static_assert(sizeof(CUtensorMap) == sizeof(wig::TensorMap), "tensor map size");
  memcpy(&h->tmap, &m, sizeof(m));
  h->tmap_W = W;
  return WIG_OK;
}

// Status word of the kernels' bounded waits: WIG_ERR_TIMEOUT (and cleared) if one gave up.
static int wig_check_status(wig_handle* h, cudaStream_t st) {
  int v = 0;
  WIG_CUDA(cudaMemcpyAsync(&v, h->status, sizeof(int), cudaMemcpyDeviceToHost, st));
  WIG_CUDA(cudaStreamSynchronize(st));
  if (v) {
    WIG_CUDA(cudaMemsetAsync(h->status, 0, sizeof(int), st));
    return fail(WIG_ERR_TIMEOUT, "a kernel's bounded wait for its tile copy gave up");
  }
  return WIG_OK;
}

static int wig_run_step(wig_handle* h, WigRunState* S, int64_t n, cudaStream_t st) {
  if (h->strang) return wig_run_step_strang(h, S, n, st);
  const int first = (S->flags & WIG_RUN_CONTINUE) ? 0 : 1;
  int mode = (n == 0) ? first : (S->damped ? 2 : 0);
  double* obs_row = h->obs + (size_t)n * WIG_NOBS;
  const bool prof = h->ev_used != 0;
  if (prof) WIG_CUDA(cudaEventRecord(h->ev[3 * n], st));
  void* xargs[] = {&S->a, &S->W, &mode, &obs_row};
  if (int rc = launch(h->f_x, h->n_cta_x, h->xnt, h->smem_x, st, xargs)) return rc;
  if (prof) WIG_CUDA(cudaEventRecord(h->ev[3 * n + 1], st));
  double t = (double)(S->t_index0 + n) * h->d.dt;
  if (h->rf) {
    if (h->tma && h->tmap_W != (const void*)S->W)
      if (int rc = encode_tile_map(h, S->W)) return rc;
    void* rargs[] = {&S->a, &S->W, &t, &h->tmap};
    if (int rc = launch(h->f_p, h->n_cta_p, h->pnt, h->smem_p, st, rargs)) return rc;
  } else {
    void* pargs[] = {&S->a, &S->W, &t};
    if (int rc = launch(h->f_p, h->n_cta_p, h->pnt, h->smem_p, st, pargs)) return rc;
  }
  if (h->odm) {
    // Lindbladian_ODM_Order1 (:1637-1643); GPU_Wigner2D_ODM2 applies a damping
    // (sign +1, weight1) then a pumping (sign -1, weight2) term (:2169-2176)
    for (int j = 0; j < h->d.n_lindblad; ++j) {
      void* oxargs[] = {&S->a, &S->W, &h->odm_T};
      if (int rc = launch(h->f_ox, h->n_cta_x, h->xnt, h->smem_odm_x, st, oxargs)) return rc;
      double coef = h->odm_coef[j], sign = h->odm_sign[j];
      void* opargs[] = {&S->a, &S->W, &h->odm_T, &coef, &sign};
      if (int rc = launch(h->f_op, h->n_cta_p, h->pnt, h->smem_odm_p, st, opargs)) return rc;
    }
  }
  if (prof) WIG_CUDA(cudaEventRecord(h->ev[3 * n + 2], st));
  S->a.n_partials = h->n_cta_p;
  return WIG_OK;
}

static int wig_run_end(wig_handle* h, WigRunState* S, cudaStream_t st) {
  int fmode = (S->n_prop == 0) ? ((S->flags & WIG_RUN_CONTINUE) ? 0 : 1) : (S->damped ? 2 : 0);
  double* last_row = h->obs + (size_t)S->n_prop * WIG_NOBS;
  void* args[] = {&S->a, &fmode, &last_row, &h->scale};
  if (int rc = launch(h->f_fin, 1, h->rnt, 0, st, args)) return rc;
  if (fmode != 0) {
    long n = (long)h->d.n_x * h->d.n_p;
    void* sargs[] = {&S->W, &n, &h->scale};
    if (int rc = launch(h->f_scale, clampi((int)(n / (4 * h->rnt)), 1, 592), h->rnt, 0, st, sargs)) return rc;
  }
  return WIG_OK;
}

static int wig_copy_obs(wig_handle* h, int64_t n_prop, double* obs_host, cudaStream_t st) {
  const size_t nobs = (size_t)(n_prop + 1) * WIG_NOBS;
  WIG_CUDA(cudaMemcpyAsync(obs_host, h->obs, nobs * sizeof(double), cudaMemcpyDeviceToHost, st));
  return WIG_OK;
}

extern "C" int wig_run(wig_handle* h, void* W_dev, int64_t t_index0, int64_t n_prop, uint32_t flags,
                       double* obs_host, void* stream) {
  if (int rc = wig_run_check(h, W_dev, n_prop)) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  WigRunState S;
  if (int rc = wig_run_begin(h, &S, W_dev, t_index0, n_prop, flags, st)) return rc;
  for (int64_t n = 0; n < n_prop; ++n)
    if (int rc = wig_run_step(h, &S, n, st)) return rc;
  if (int rc = wig_run_end(h, &S, st)) return rc;
  h->psq_n = n_prop;
  h->last_stream = st;
  if (obs_host) {
    if (int rc = wig_copy_obs(h, n_prop, obs_host, st)) return rc;
    WIG_CUDA(cudaStreamSynchronize(st));
    if (h->tma)
      if (int rc = wig_check_status(h, st)) return rc;
    return check_finite(obs_host, (size_t)(n_prop + 1) * WIG_NOBS, "wig_run observables");
  }
  return WIG_OK;
}

// ------------------------------------------------------------------ Bloch (imaginary time)
// GPU_Wigner2D_GPitaevskii_Bloch.Run / Run_ExitedState1 (:2105-2545): the device
// work of one step; the host keeps the reference's accept / reject and
// step-halving logic.
static int bloch_check(wig_handle* h, void* W_dev, double* stats, const char* what) {
  if (!h || !W_dev || !stats) return fail(WIG_ERR_ARG, "%s: null argument", what);
  if (!h->strang) return fail(WIG_ERR_ARG, "%s: the handle needs splitting = WIG_SPLIT_STRANG_GP", what);
  if (((uintptr_t)W_dev & 15) != 0) return fail(WIG_ERR_ARG, "%s: W must be 16-byte aligned", what);
  int cur;
  WIG_CUDA(cudaGetDevice(&cur));
  if (cur != h->device) return fail(WIG_ERR_ARG, "%s: current device %d != handle device %d", what, cur, h->device);
  return WIG_OK;
}

// sums[NBL] over the grid (CTA partials summed on the host in CTA order)
static int bloch_sums(wig_handle* h, double2* W, const double2* W0, double* sums, cudaStream_t st) {
  void* args[] = {&h->a, &W, &W0, &h->bloch_part};
  if (int rc = launch(h->f_br, h->n_cta_r, h->rnt, 0, st, args)) return rc;
  std::vector<double> part((size_t)h->n_cta_r * wig::NBL);
  WIG_CUDA(cudaMemcpyAsync(part.data(), h->bloch_part, part.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
  WIG_CUDA(cudaStreamSynchronize(st));
  for (int v = 0; v < wig::NBL; ++v) sums[v] = 0.;
  for (int c = 0; c < h->n_cta_r; ++c)
    for (int v = 0; v < wig::NBL; ++v) sums[v] += part[(size_t)c * wig::NBL + v];
  return WIG_OK;
}

static int bloch_axpy(wig_handle* h, double2* W, const double2* W0, double2 c, double2 s, cudaStream_t st) {
  long n = (long)h->d.n_x * h->d.n_p;
  void* args[] = {&W, &W0, &n, &c, &s};
  return launch(h->f_ba, clampi((int)(n / (4 * h->rnt)), 1, 592), h->rnt, 0, st, args);
}

static double2 cdiv1(double2 z) {   // 1 / z (Smith)
  double2 r;
  if (fabs(z.x) >= fabs(z.y)) {
    const double rat = z.y / z.x, scl = 1.0 / (z.x + z.y * rat);
    r.x = scl; r.y = -rat * scl;
  } else {
    const double rat = z.x / z.y, scl = 1.0 / (z.y + z.x * rat);
    r.x = rat * scl; r.y = -scl;
  }
  return r;
}

// stats of the (normalised) W: [0..4] <x>, <x^2>, <p>, <p^2>, <K(p) + V(0, x)>;
// [5, 6] purity 2 pi hbar dXdP sum W^2; [7] mean-field energy 0.5 a_GP sum_x P^2 dx;
// [8] 1 if a row sum (p-marginal) is negative (with_marginal), else 0; [9] the
// norm dXdP sum W before normalisation (Re).
static int bloch_stats_of(wig_handle* h, double2* W, bool with_marginal, double* stats, cudaStream_t st) {
  double sums[wig::NBL];
  if (int rc = bloch_sums(h, W, nullptr, sums, st)) return rc;
  const double dXdP = h->a.dX * h->a.dP;
  for (int k = 0; k < 5; ++k) stats[k] = dXdP * sums[2 + k];
  const double pf = 2. * M_PI * h->d.hbar * dXdP;
  stats[5] = pf * sums[7];
  stats[6] = pf * sums[8];
  stats[7] = 0.;
  if (h->gp) {
    const int NX = h->d.n_x, NP = h->d.n_p, cnt = NX < 256 ? NX : 256;
    void* cargs[] = {&W, &h->gp_chunks};
    if (int rc = launch2d(h->f_gcs, (unsigned)(NX / cnt), (unsigned)(NP / 16), (unsigned)cnt, 0, st, cargs)) return rc;
    int nch = h->n_chunks, zero = 0;
    double* psq_d = h->bloch_psq;
    void* margs[] = {&h->a, &h->gp_chunks, &nch, &zero, &h->gp_P, &psq_d};
    if (int rc = launch(h->f_gm, 1, 256, 0, st, margs)) return rc;
    double psq_h = 0.;
    WIG_CUDA(cudaMemcpyAsync(&psq_h, psq_d, sizeof(double), cudaMemcpyDeviceToHost, st));
    WIG_CUDA(cudaStreamSynchronize(st));
    stats[7] = 0.5 * h->d.gp_coefficient * psq_h;   // NonLinearEnergy (:1757-1758)
  }
  stats[8] = 0.;
  if (with_marginal) {
    void* rargs[] = {&W, &h->rowsums};
    if (int rc = launch(h->f_rs, h->d.n_p, 256, 0, st, rargs)) return rc;
    std::vector<double2> rows(h->d.n_p);
    WIG_CUDA(cudaMemcpyAsync(rows.data(), h->rowsums, rows.size() * sizeof(double2), cudaMemcpyDeviceToHost, st));
    WIG_CUDA(cudaStreamSynchronize(st));
    for (const double2& r : rows)
      if (r.x * h->a.dX < 0.) { stats[8] = 1.; break; }
  }
  return WIG_OK;
}

// divide W by norm = sum W * c0 (c0 = dX dP applied as (S dX) dP when initial, S (dX dP) per step)
static int bloch_normalise(wig_handle* h, double2* W, bool initial, double* norm_re, cudaStream_t st) {
  double sums[wig::NBL];
  if (int rc = bloch_sums(h, W, nullptr, sums, st)) return rc;
  double2 S = make_double2(sums[0], sums[1]), nrm;
  if (initial) nrm = make_double2(S.x * h->a.dX * h->a.dP, S.y * h->a.dX * h->a.dP);
  else { const double d = h->a.dX * h->a.dP; nrm = make_double2(S.x * d, S.y * d); }
  *norm_re = nrm.x;
  return bloch_axpy(h, W, nullptr, make_double2(0., 0.), cdiv1(nrm), st);
}

extern "C" int wig_bloch_stats(wig_handle* h, void* W_dev, int32_t normalise, double* stats, void* stream) {
  if (int rc = bloch_check(h, W_dev, stats, "wig_bloch_stats")) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  double2* W = (double2*)W_dev;
  double nre = 0.;
  if (normalise)
    if (int rc = bloch_normalise(h, W, true, &nre, st)) return rc;
  if (int rc = bloch_stats_of(h, W, false, stats, st)) return rc;
  stats[9] = nre;
  return check_finite(stats, WIG_BLOCH_NSTATS, "wig_bloch_stats");
}

extern "C" int wig_bloch_step(wig_handle* h, void* W_dev, int64_t t_index, double dtb, const void* W0_dev,
                              double* stats, void* stream) {
  if (int rc = bloch_check(h, W_dev, stats, "wig_bloch_step")) return rc;
  if (!(dtb > 0.) || !std::isfinite(dtb)) return fail(WIG_ERR_ARG, "wig_bloch_step: dtb must be > 0");
  if (W0_dev && ((uintptr_t)W0_dev & 15) != 0) return fail(WIG_ERR_ARG, "wig_bloch_step: W0 must be 16-byte aligned");
  cudaStream_t st = (cudaStream_t)stream;
  double2* W = (double2*)W_dev;
  const double2* W0 = (const double2*)W0_dev;
  const double t = (double)t_index * h->d.dt;
  const int NX = h->d.n_x, NP = h->d.n_p, cnt = NX < 256 ? NX : 256;
  auto gexp = [&](double** out) -> int {   // mean-field exponent of the current W
    *out = nullptr;
    if (!h->gp) return WIG_OK;
    void* cargs[] = {&W, &h->gp_chunks};
    if (int rc = launch2d(h->f_gcs, (unsigned)(NX / cnt), (unsigned)(NP / 16), (unsigned)cnt, 0, st, cargs)) return rc;
    int nch = h->n_chunks, zero = 0;
    double* nopsq = nullptr;
    void* margs[] = {&h->a, &h->gp_chunks, &nch, &zero, &h->gp_P, &nopsq};
    if (int rc = launch(h->f_gm, 1, 256, 0, st, margs)) return rc;
    double dt_ = dtb;
    void* gargs[] = {&h->a, &h->gp_P, &dt_, &h->gp_phase};
    if (int rc = launch(h->f_gb, h->n_cta_x, h->xnt, h->smem_gph, st, gargs)) return rc;
    *out = h->gp_phase;
    return WIG_OK;
  };
  double* ge = nullptr;
  double tt = t, dd = dtb;
  if (int rc = gexp(&ge)) return rc;
  {
    void* args[] = {&h->a, &W, &tt, &dd, &ge};
    if (int rc = launch(h->f_bph, h->n_cta_p, h->pnt, h->smem_ph, st, args)) return rc;
  }
  {
    void* args[] = {&h->a, &W, &dd};
    if (int rc = launch(h->f_bx, h->n_cta_x, h->xnt, h->smem_x, st, args)) return rc;
  }
  if (int rc = gexp(&ge)) return rc;
  {
    void* args[] = {&h->a, &W, &tt, &dd, &ge};
    if (int rc = launch(h->f_bph, h->n_cta_p, h->pnt, h->smem_ph, st, args)) return rc;
  }
  if (W0) {
    // Run_ExitedState1 (:2429-2434): W -= c W0, c = 2 pi hbar dXdP sum W W0
    double sums[wig::NBL];
    if (int rc = bloch_sums(h, W, W0, sums, st)) return rc;
    const double pf = 2. * M_PI * h->d.hbar * h->a.dX * h->a.dP;
    if (int rc = bloch_axpy(h, W, W0, make_double2(pf * sums[9], pf * sums[10]), make_double2(1., 0.), st)) return rc;
  }
  double nre = 0.;
  if (int rc = bloch_normalise(h, W, false, &nre, st)) return rc;
  if (int rc = bloch_stats_of(h, W, W0 != nullptr, stats, st)) return rc;
  stats[9] = nre;
  return check_finite(stats, WIG_BLOCH_NSTATS, "wig_bloch_step");
}

extern "C" int wig_run_probability_square(wig_handle* h, double* out, int64_t n) {
  if (!h || !out || n < 0) return fail(WIG_ERR_ARG, "wig_run_probability_square: bad arguments");
  if (!h->gp) return fail(WIG_ERR_ARG, "wig_run_probability_square: the handle has no Gross-Pitaevskii term");
  if (n > h->psq_n) return fail(WIG_ERR_ARG, "wig_run_probability_square: %lld values asked, the last run made %lld",
                                (long long)n, (long long)h->psq_n);
  WIG_CUDA(cudaStreamSynchronize(h->last_stream));
  if (n) WIG_CUDA(cudaMemcpy(out, h->psq, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost));
  return WIG_OK;
}

extern "C" int wig_run_many(wig_handle* const* hs, void* const* Ws, int64_t count, int64_t t_index0,
                            int64_t n_prop, uint32_t flags, double* const* obs_host, void* stream) {
  if (!hs || !Ws || count < 1) return fail(WIG_ERR_ARG, "wig_run_many: empty batch");
  for (int64_t i = 0; i < count; ++i) {
    if (int rc = wig_run_check(hs[i], Ws[i], n_prop)) return rc;
    for (int64_t j = 0; j < i; ++j)
      if (hs[j] == hs[i]) return fail(WIG_ERR_ARG, "wig_run_many: a handle appears twice");
  }
  cudaStream_t st = (cudaStream_t)stream;
  std::vector<WigRunState> S((size_t)count);
  for (int64_t i = 0; i < count; ++i)
    if (int rc = wig_run_begin(hs[i], &S[i], Ws[i], t_index0, n_prop, flags, st)) return rc;
  for (int64_t n = 0; n < n_prop; ++n)
    for (int64_t i = 0; i < count; ++i)
      if (int rc = wig_run_step(hs[i], &S[i], n, st)) return rc;
  for (int64_t i = 0; i < count; ++i)
    if (int rc = wig_run_end(hs[i], &S[i], st)) return rc;
  if (obs_host) {
    for (int64_t i = 0; i < count; ++i)
      if (obs_host[i])
        if (int rc = wig_copy_obs(hs[i], n_prop, obs_host[i], st)) return rc;
    WIG_CUDA(cudaStreamSynchronize(st));
    for (int64_t i = 0; i < count; ++i)
      if (obs_host[i])
        if (int rc = check_finite(obs_host[i], (size_t)(n_prop + 1) * WIG_NOBS, "wig_run_many observables"))
          return rc;
  }
  return WIG_OK;
}

extern "C" int wig_profile(wig_handle* h, double* ms_out, int64_t* launches) {
  if (!h || !ms_out) return fail(WIG_ERR_ARG, "wig_profile: null argument");
  ms_out[0] = ms_out[1] = 0.;
  const size_t steps = h->ev_used / 3;
  for (size_t n = 0; n < steps; ++n) {
    float a = 0.f, b = 0.f;
    WIG_CUDA(cudaEventSynchronize(h->ev[3 * n + 2]));
    WIG_CUDA(cudaEventElapsedTime(&a, h->ev[3 * n], h->ev[3 * n + 1]));
    WIG_CUDA(cudaEventElapsedTime(&b, h->ev[3 * n + 1], h->ev[3 * n + 2]));
    ms_out[0] += a;
    ms_out[1] += b;
  }
  if (launches) *launches = (int64_t)steps;
  return WIG_OK;
}

extern "C" int wig_run_host(wig_handle* h, const void* W_in, void* W_out, int64_t t_index0, int64_t n_prop,
                            uint32_t flags, double* obs_host, void* stream) {
  if (!h || !W_in || !W_out) return fail(WIG_ERR_ARG, "wig_run_host: null argument");
  const size_t bytes = (size_t)h->d.n_x * h->d.n_p * sizeof(double2);
  if (!h->W_host_stage) {
    void* p = nullptr;
    WIG_CUDA(cudaMalloc(&p, bytes));
    h->W_host_stage = (double2*)p;
  }
  cudaStream_t st = (cudaStream_t)stream;
  WIG_CUDA(cudaMemcpyAsync(h->W_host_stage, W_in, bytes, cudaMemcpyHostToDevice, st));
  int rc = wig_run(h, h->W_host_stage, t_index0, n_prop, flags, nullptr, stream);
  if (rc) return rc;
  WIG_CUDA(cudaMemcpyAsync(W_out, h->W_host_stage, bytes, cudaMemcpyDeviceToHost, st));
  const size_t nobs = (size_t)(n_prop + 1) * WIG_NOBS;
  if (obs_host) WIG_CUDA(cudaMemcpyAsync(obs_host, h->obs, nobs * sizeof(double), cudaMemcpyDeviceToHost, st));
  WIG_CUDA(cudaStreamSynchronize(st));
  if (obs_host) return check_finite(obs_host, nobs, "wig_run_host observables");
  return WIG_OK;
}

extern "C" int wig_destroy(wig_handle* h) {
  if (!h) return WIG_OK;
  cudaDeviceSynchronize();
  for (cudaEvent_t e : h->ev) cudaEventDestroy(e);
  h->bufs.free_all();
  if (h->obs) cudaFree(h->obs);
  if (h->W_host_stage) cudaFree(h->W_host_stage);
  delete h;
  return WIG_OK;
}

// ======================================================================== Dirac
struct dirac_handle {
  int device = 0;
  dirac_desc d{};
  wig::DiracArgs a{};
  CUfunction f_row = nullptr, f_col = nullptr, f_fin = nullptr, f_scale = nullptr;
  int rows = 1, rnt = 256, cc = 1, cnt = 256, snt = 256;
  int n_row = 1, n_col = 1, smem_row = 0, smem_col = 0;
  DevBuf bufs;
  double* obs = nullptr;
  size_t obs_cap = 0;
  double2* scale = nullptr;
  double2* psi_host_stage = nullptr;
};

struct DiracPlan {
  int rows, rnt, rmb, cc, cnt, cmb, snt, n_row, n_col, smem_row, smem_col;
  double dX, dY, Pxa, Pya, dPx, dPy;
  std::string src;
};

static int dirac_plan(const dirac_desc* d, DiracPlan* P) {
  if (!d) return fail(WIG_ERR_ARG, "dirac: null descriptor");
  if (d->abi_version != WIG_ABI_VERSION)
    return fail(WIG_ERR_ARG, "dirac: abi_version %d != %d", d->abi_version, WIG_ABI_VERSION);
  if (!pow2_in_range(d->n_x) || !pow2_in_range(d->n_y) || d->n_x > 2048 || d->n_y > 2048)
    return fail(WIG_ERR_ARG, "grid %d x %d: n_x and n_y must be powers of two in [16, 2048]", d->n_x, d->n_y);
  if (!(d->x_amplitude > 0) || !(d->y_amplitude > 0) || !std::isfinite(d->dt) || !std::isfinite(d->c))
    return fail(WIG_ERR_ARG, "amplitudes must be > 0, dt and c finite");
  if (d->constants != WIG_CONST_CUDA_F && d->constants != WIG_CONST_EXACT)
    return fail(WIG_ERR_ARG, "unknown constants mode %d", d->constants);
  if (d->precision != WIG_PREC_C128) return fail(WIG_ERR_UNSUPPORTED, "precision %d not available", d->precision);
  const std::string A0 = expr_or(d->a0, "0."), A1 = expr_or(d->a1, "0."), A2 = expr_or(d->a2, "0."),
                    A3 = expr_or(d->a3, "0.");
  if (!safe_expr(A0) || !safe_expr(A1) || !safe_expr(A2) || !safe_expr(A3))
    return fail(WIG_ERR_ARG, "expression strings may not contain ; { } # quotes or unbalanced ()");
  const int NX = d->n_x, NY = d->n_y, cm = d->constants;
  // ---- tiling (defaults; WIG_DIRAC_TILING="rows,rnt,rmb,cc,cnt,cmb" overrides for tuning runs)
  // One CTA transforms the 4 components of `rows` rows (or `cc` columns) of at most 512 points
  // each.  Resident CTAs per SM follow the radix-8 butterflies a thread holds per stage (1 up to
  // 512-point sequences): 3 row-pass / 4 column-pass CTAs of 256 threads per SM (80 / 64
  // registers) for one, 2 for two, 1 beyond (measured at 512^2: 1.25 -> 1.07 ms per
  // 16-replica step against 1 CTA of 2 columns).
  P->rows = clampi(512 / NX, 1, NY);
  P->rnt = round_warp(clampi(4 * P->rows * NX / 8, 32, 256));
  const int rper = (4 * P->rows * NX / 8 + P->rnt - 1) / P->rnt;
  P->rmb = rper == 1 ? 3 : (rper == 2 ? 2 : 1);
  P->cc = clampi(512 / NY, 1, NX);
  P->cnt = round_warp(clampi(4 * P->cc * NY / 8, 32, 256));
  const int cper = (4 * P->cc * NY / 8 + P->cnt - 1) / P->cnt;
  P->cmb = cper == 1 ? 4 : (cper == 2 ? 2 : 1);
  if (const char* tv = getenv("WIG_DIRAC_TILING")) {
    int v[6];
    if (sscanf(tv, "%d,%d,%d,%d,%d,%d", &v[0], &v[1], &v[2], &v[3], &v[4], &v[5]) == 6) {
      if (v[0] > 0) P->rows = clampi(v[0], 1, NY);
      if (v[1] > 0) P->rnt = round_warp(clampi(v[1], 32, 1024));
      if (v[2] > 0) P->rmb = v[2];
      if (v[3] > 0) P->cc = clampi(v[3], 1, NX);
      if (v[4] > 0) P->cnt = round_warp(clampi(v[4], 32, 1024));
      if (v[5] > 0) P->cmb = v[5];
    }
  }
  if ((NY % P->rows) != 0 || (NX % P->cc) != 0)
    return fail(WIG_ERR_ARG, "dirac tiling: %d rows / %d columns per CTA must divide the grid", P->rows, P->cc);
  P->snt = 256;
  P->n_row = NY / P->rows;
  P->n_col = NX / P->cc;
  P->smem_row = wig::padded_size(4 * P->rows * NX) * (int)sizeof(double2);
  P->smem_col = wig::padded_size(4 * P->cc * NY) * (int)sizeof(double2);
  // GPU_Dirac2D.py:312-346
  P->dX = 2. * d->x_amplitude / (double)NX;
  P->dY = 2. * d->y_amplitude / (double)NY;
  P->Pxa = M_PI / P->dX;
  P->Pya = M_PI / P->dY;
  P->dPx = 2 * P->Pxa / NX;
  P->dPy = 2 * P->Pya / NY;
  struct { const char* name; double v; } consts[] = {{"mass", d->mass}, {"c", d->c}, {"dt", d->dt},
                                                      {"dX", P->dX},    {"dY", P->dY}, {"dPx", P->dPx},
                                                      {"dPy", P->dPy}};
  std::string src = kMathPrelude;
  for (auto& c : consts) src += "__constant__ double " + std::string(c.name) + "=" + fmt_const(c.v, cm) + ";";
  src += "\nstruct UserPhys {\n  double cf[8];\n";
  const std::string* As[4] = {&A0, &A1, &A2, &A3};
  for (int i = 0; i < 4; ++i)
    src += "  __device__ __forceinline__ double A" + std::to_string(i) +
           "(double t, double x, double y) const { return (" + *As[i] + "); }\n";
  src += "};\n";
  char macros[512];
  snprintf(macros, sizeof(macros),
           "#define DIR_NX %d\n#define DIR_NY %d\n#define DIR_ROWS %d\n#define DIR_RNT %d\n#define DIR_RMB %d\n"
           "#define DIR_C %d\n#define DIR_CNT %d\n#define DIR_CMB %d\n#define DIR_SNT %d\n",
           NX, NY, P->rows, P->rnt, P->rmb, P->cc, P->cnt, P->cmb, P->snt);
  src += macros;
  src += kJitDiracSource;
  P->src.swap(src);
  return WIG_OK;
}

extern "C" int dirac_jit_check(const dirac_desc* d, char* log, int64_t log_cap) {
  DiracPlan P;
  if (int rc = dirac_plan(d, &P)) { copy_log(g_last_error, log, log_cap); return rc; }
  std::lock_guard<std::mutex> lk(g_mu);
  std::vector<char> cubin;
  std::string lg;
  int rc = nvrtc_compile(P.src, &cubin, &lg, true);
  copy_log(rc ? g_last_error : lg, log, log_cap);
  return rc;
}

extern "C" int dirac_create(const dirac_desc* d, dirac_handle** out) {
  if (!out) return fail(WIG_ERR_ARG, "dirac_create: null argument");
  *out = nullptr;
  DiracPlan P;
  if (int rc = dirac_plan(d, &P)) return rc;
  int device = 0;
  WIG_CUDA(cudaGetDevice(&device));
  WIG_CUDA(cudaFree(0));
  dirac_handle* h = new dirac_handle();
  h->d = *d;
  h->device = device;
  const int NX = d->n_x, NY = d->n_y, cm = d->constants;
  h->rows = P.rows; h->rnt = P.rnt; h->cc = P.cc; h->cnt = P.cnt; h->snt = P.snt;
  h->n_row = P.n_row; h->n_col = P.n_col; h->smem_row = P.smem_row; h->smem_col = P.smem_col;
  const double dX = P.dX, dY = P.dY, Pxa = P.Pxa, Pya = P.Pya, dPx = P.dPx, dPy = P.dPy;
  const std::string& src = P.src;
  CUmodule mod;
  int rc = get_module(src, h->device, &mod);
  if (!rc) rc = get_fn(mod, "dirac_rowpass", &h->f_row, h->smem_row);
  if (!rc) rc = get_fn(mod, "dirac_colpass", &h->f_col, h->smem_col);
  if (!rc) rc = get_fn(mod, "dirac_final", &h->f_fin, 0);
  if (!rc) rc = get_fn(mod, "dirac_scale", &h->f_scale, 0);
  CUfunction f_setup = nullptr;
  if (!rc) rc = get_fn(mod, "dirac_setup", &f_setup, 0);
  if (rc) { delete h; return rc; }

  wig::DiracArgs& a = h->a;
  a.mass = kval(d->mass, cm); a.c = kval(d->c, cm); a.dt = kval(d->dt, cm);
  a.dX = kval(dX, cm); a.dY = kval(dY, cm); a.dPx = kval(dPx, cm); a.dPy = kval(dPy, cm);
  a.dX_e = dX; a.dY_e = dY; a.dPx_e = dPx; a.dPy_e = dPy; a.mass_e = d->mass; a.c_e = d->c;
  std::vector<double> xt = d->x_table ? std::vector<double>(d->x_table, d->x_table + NX) : shifted_range(d->x_amplitude, NX);
  std::vector<double> yt = d->y_table ? std::vector<double>(d->y_table, d->y_table + NY) : shifted_range(d->y_amplitude, NY);
  std::vector<double> pxt = d->px_table ? std::vector<double>(d->px_table, d->px_table + NX) : shifted_range(Pxa, NX);
  std::vector<double> pyt = d->py_table ? std::vector<double>(d->py_table, d->py_table + NY) : shifted_range(Pya, NY);
  std::vector<double2> twx = twiddles(NX), twy = twiddles(NY);
  double *x_d, *y_d, *px_d, *py_d, *bx_d, *by_d, *pr0, *pr1, *pc;
  double2 *twx_d, *twy_d;
  DevBuf& B = h->bufs;
  rc = B.alloc(&x_d, NX, xt.data());
  if (!rc) rc = B.alloc(&y_d, NY, yt.data());
  if (!rc) rc = B.alloc(&px_d, NX, pxt.data());
  if (!rc) rc = B.alloc(&py_d, NY, pyt.data());
  if (!rc) rc = B.alloc(&bx_d, 2 * (size_t)NX);
  if (!rc) rc = B.alloc(&by_d, 2 * (size_t)NY);
  if (!rc) rc = B.alloc(&twx_d, NX, twx.data());
  if (!rc) rc = B.alloc(&twy_d, NY, twy.data());
  if (!rc) rc = B.alloc(&pr0, (size_t)h->n_row * wig::DNR);
  if (!rc) rc = B.alloc(&pr1, (size_t)h->n_row * wig::DNR);
  if (!rc) rc = B.alloc(&pc, (size_t)h->n_col * wig::DNC);
  if (!rc) rc = B.alloc(&h->scale, 1);
  if (rc) { B.free_all(); delete h; return rc; }
  a.x_tab = x_d; a.y_tab = y_d; a.px_tab = px_d; a.py_tab = py_d; a.bx = bx_d; a.by = by_d;
  a.tw_x = twx_d; a.tw_y = twy_d; a.part_row[0] = pr0; a.part_row[1] = pr1; a.part_col = pc;
  a.n_row_cta = h->n_row; a.n_col_cta = h->n_col;
  for (int i = 0; i < 8; ++i) a.coef[i] = d->coef[i];
  {
    void* args[] = {&bx_d, &by_d};
    rc = launch(f_setup, 8, 256, 0, 0, args);
    if (!rc) {
      cudaError_t e = cudaDeviceSynchronize();
      if (e != cudaSuccess) rc = fail(WIG_ERR_CUDA, "dirac_setup: %s", cudaGetErrorString(e));
    }
    if (rc) { B.free_all(); delete h; return rc; }
  }
  *out = h;
  return WIG_OK;
}

struct DiracRunState {
  wig::DiracArgs a;
  double2* psi;
  int64_t t_index0, n_steps;
};

static int dirac_run_check(dirac_handle* h, void* psi_dev, int64_t n_steps) {
  if (!h || !psi_dev) return fail(WIG_ERR_ARG, "dirac_run: null handle or psi");
  if (((uintptr_t)psi_dev & 15) != 0) return fail(WIG_ERR_ARG, "dirac_run: psi must be 16-byte aligned");
  if (n_steps < 1) return fail(WIG_ERR_ARG, "dirac_run: n_steps must be >= 1");
  int cur;
  WIG_CUDA(cudaGetDevice(&cur));
  if (cur != h->device) return fail(WIG_ERR_ARG, "dirac_run: current device %d != handle device %d", cur, h->device);
  return ensure_obs(&h->obs, &h->obs_cap, (size_t)n_steps * DIRAC_NOBS);
}

static int dirac_run_begin(dirac_handle* h, DiracRunState* S, void* psi_dev, int64_t t_index0, int64_t n_steps,
                           cudaStream_t st) {
  S->a = h->a;
  S->psi = (double2*)psi_dev;
  S->t_index0 = t_index0;
  S->n_steps = n_steps;
  int mode = 0, parity = 0;
  double t_step = 0., t_obs = h->d.dt * (double)(t_index0 + 1);
  double* obs_row = nullptr;
  void* args[] = {&S->a, &S->psi, &mode, &parity, &t_step, &t_obs, &obs_row};
  return launch(h->f_row, h->n_row, h->rnt, h->smem_row, st, args);
}

static int dirac_run_step(dirac_handle* h, DiracRunState* S, int64_t n, cudaStream_t st) {
  void* cargs[] = {&S->a, &S->psi};
  if (int rc = launch(h->f_col, h->n_col, h->cnt, h->smem_col, st, cargs)) return rc;
  const double dt = h->d.dt;
  int mode = (n == S->n_steps - 1) ? 2 : 1, parity = (int)((n + 1) & 1);
  double t_step = dt * (double)(S->t_index0 + n + 1), t_obs = dt * (double)(S->t_index0 + n + 2);
  double* obs_row = h->obs + (size_t)n * DIRAC_NOBS;
  void* args[] = {&S->a, &S->psi, &mode, &parity, &t_step, &t_obs, &obs_row};
  return launch(h->f_row, h->n_row, h->rnt, h->smem_row, st, args);
}

static int dirac_run_end(dirac_handle* h, DiracRunState* S, cudaStream_t st) {
  int parity = (int)(S->n_steps & 1);
  void* args[] = {&S->a, &parity, &h->scale};
  if (int rc = launch(h->f_fin, 1, h->snt, 0, st, args)) return rc;
  long n = 4L * h->d.n_x * h->d.n_y;
  void* sargs[] = {&S->psi, &n, &h->scale};
  return launch(h->f_scale, clampi((int)(n / (4 * h->snt)), 1, 592), h->snt, 0, st, sargs);
}

extern "C" int dirac_run(dirac_handle* h, void* psi_dev, int64_t t_index0, int64_t n_steps, double* obs_host,
                         void* stream) {
  if (int rc = dirac_run_check(h, psi_dev, n_steps)) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  DiracRunState S;
  if (int rc = dirac_run_begin(h, &S, psi_dev, t_index0, n_steps, st)) return rc;
  for (int64_t n = 0; n < n_steps; ++n)
    if (int rc = dirac_run_step(h, &S, n, st)) return rc;
  if (int rc = dirac_run_end(h, &S, st)) return rc;
  if (obs_host) {
    const size_t nobs = (size_t)n_steps * DIRAC_NOBS;
    WIG_CUDA(cudaMemcpyAsync(obs_host, h->obs, nobs * sizeof(double), cudaMemcpyDeviceToHost, st));
    WIG_CUDA(cudaStreamSynchronize(st));
    return check_finite(obs_host, nobs, "dirac_run observables");
  }
  return WIG_OK;
}

extern "C" int dirac_run_many(dirac_handle* const* hs, void* const* psis, int64_t count, int64_t t_index0,
                              int64_t n_steps, double* const* obs_host, void* stream) {
  if (!hs || !psis || count < 1) return fail(WIG_ERR_ARG, "dirac_run_many: empty batch");
  for (int64_t i = 0; i < count; ++i) {
    if (int rc = dirac_run_check(hs[i], psis[i], n_steps)) return rc;
    for (int64_t j = 0; j < i; ++j)
      if (hs[j] == hs[i]) return fail(WIG_ERR_ARG, "dirac_run_many: a handle appears twice");
  }
  cudaStream_t st = (cudaStream_t)stream;
  std::vector<DiracRunState> S((size_t)count);
  for (int64_t i = 0; i < count; ++i)
    if (int rc = dirac_run_begin(hs[i], &S[i], psis[i], t_index0, n_steps, st)) return rc;
  for (int64_t n = 0; n < n_steps; ++n)
    for (int64_t i = 0; i < count; ++i)
      if (int rc = dirac_run_step(hs[i], &S[i], n, st)) return rc;
  for (int64_t i = 0; i < count; ++i)
    if (int rc = dirac_run_end(hs[i], &S[i], st)) return rc;
  if (obs_host) {
    const size_t nobs = (size_t)n_steps * DIRAC_NOBS;
    for (int64_t i = 0; i < count; ++i)
      if (obs_host[i])
        WIG_CUDA(cudaMemcpyAsync(obs_host[i], hs[i]->obs, nobs * sizeof(double), cudaMemcpyDeviceToHost, st));
    WIG_CUDA(cudaStreamSynchronize(st));
    for (int64_t i = 0; i < count; ++i)
      if (obs_host[i])
        if (int rc = check_finite(obs_host[i], nobs, "dirac_run_many observables")) return rc;
  }
  return WIG_OK;
}

extern "C" int dirac_run_host(dirac_handle* h, const void* psi_in, void* psi_out, int64_t t_index0,
                              int64_t n_steps, double* obs_host, void* stream) {
  if (!h || !psi_in || !psi_out) return fail(WIG_ERR_ARG, "dirac_run_host: null argument");
  const size_t bytes = 4 * (size_t)h->d.n_x * h->d.n_y * sizeof(double2);
  if (!h->psi_host_stage) {
    void* p = nullptr;
    WIG_CUDA(cudaMalloc(&p, bytes));
    h->psi_host_stage = (double2*)p;
  }
  cudaStream_t st = (cudaStream_t)stream;
  WIG_CUDA(cudaMemcpyAsync(h->psi_host_stage, psi_in, bytes, cudaMemcpyHostToDevice, st));
  int rc = dirac_run(h, h->psi_host_stage, t_index0, n_steps, nullptr, stream);
  if (rc) return rc;
  WIG_CUDA(cudaMemcpyAsync(psi_out, h->psi_host_stage, bytes, cudaMemcpyDeviceToHost, st));
  const size_t nobs = (size_t)n_steps * DIRAC_NOBS;
  if (obs_host) WIG_CUDA(cudaMemcpyAsync(obs_host, h->obs, nobs * sizeof(double), cudaMemcpyDeviceToHost, st));
  WIG_CUDA(cudaStreamSynchronize(st));
  if (obs_host) return check_finite(obs_host, nobs, "dirac_run_host observables");
  return WIG_OK;
}

extern "C" int dirac_destroy(dirac_handle* h) {
  if (!h) return WIG_OK;
  cudaDeviceSynchronize();
  h->bufs.free_all();
  if (h->obs) cudaFree(h->obs);
  if (h->psi_host_stage) cudaFree(h->psi_host_stage);
  delete h;
  return WIG_OK;
}

extern "C" const char* wig_last_error(void) { return g_last_error.c_str(); }

// Records a failure for wig_last_error from other translation units of the library.
int wig_record_error(int code, const char* msg) { return fail(code, "%s", msg); }
extern "C" int wig_abi_version(void) { return WIG_ABI_VERSION; }

// ======================================================================== batched form
// Many independent Wigner2D instances (polynomial potentials, uneven grids) in
// one x-pass and one p-pass launch per step, real FP32 storage, FP32 or mixed
// (FP64 kinetic / Moyal) transforms; see wig_batch.cuh.  A run can be
// captured once into a CUDA graph (WIG_RUN_GRAPH) and replayed; the tile shape
// (warps per CTA) is chosen by wigb_autotune from timed candidates.
namespace {

struct BVariant {
  int warps = 0;
  CUfunction fx = nullptr, fp = nullptr, fr = nullptr, fs = nullptr;
  int smem_x = 0, smem_p = 0, occ_x = 1, occ_p = 1;
};

// Whether the x-pass stages its rows in shared memory (WIGB_XSTAGE).  Off by
// default.  At the register caps below, the staging buffer is what limits the
// x-pass's resident warps (a 2-warp mixed CTA: 33 KB of exchange + 16 KB of
// staging, 4 CTAs per SM); without it the x-pass runs 12 (mixed) or 16 (FP32)
// warps per SM.  On the 64-instance mixed-grid batch (B200, CUDA events): mixed
// x-pass 253 us staged at 8 warps per SM, 220 us direct at 12; FP32 173 us staged
// at 12, 164 us direct at 16.  (At the earlier 8 / 12-warp caps staging had been
// the faster one: 272 -> 240 and 182 -> 169 us.)  Tuning override (read per
// compile): WIG_BATCH_XSTAGE=0|1.
int batch_xstage(int) {
  const char* e = getenv("WIG_BATCH_XSTAGE");
  if (e && *e) return atoi(e) ? 1 : 0;
  return 0;
}

// the x-pass's exchange regions and row staging buffer (wigb_xpass: the largest size class's each)
int batch_smem_x(const std::vector<int>& classes, int warps, int prec, int xstage) {
  int ex = 0, st = 0;
  for (int n : classes) {
    ex = std::max(ex, wig::bx_exch(n, warps, prec));
    st = std::max(st, wig::bx_stage(n, warps));
  }
  return ex * (int)sizeof(float2) + (xstage ? st * (int)sizeof(float) : 0);
}
int batch_smem_p(int n, int warps) { return wig::bp_smem(n, warps) * (int)sizeof(float2); }

}  // namespace


struct wigb_handle {
  int device = 0, count = 0, n_sm = 148;
  int precision = WIGB_PREC_F32;
  std::vector<wigb_instance> inst;
  std::vector<wig::BInst> binst;
  std::vector<int> classes;
  int64_t total = 0;
  std::vector<int64_t> offsets;
  wig::BArgs a{};
  int n_xitems = 0, n_pitems = 0, grid_x = 1, grid_p = 1;
  DevBuf bufs;                      // tables that do not depend on the tile shape
  void* items_d = nullptr;          // x-items then p-items (int2), per tile shape
  double* partials_d = nullptr;
  std::map<int, BVariant> variants; // by warps per CTA
  int warps = 0;
  double* obs = nullptr;
  size_t obs_cap = 0;
  cudaGraphExec_t gexec = nullptr;  // cached graph of the last WIG_RUN_GRAPH run
  void* g_W = nullptr;
  int64_t g_t0 = -1, g_n = -1;
  uint32_t g_flags = 0;
  int g_warps = -1;
  void* g_stream = nullptr;
  std::vector<cudaEvent_t> ev;      // WIG_RUN_PROFILE (non-graph runs): 3 events per step
  size_t ev_used = 0;
  void* flush = nullptr;            // WIG_RUN_FLUSH_L2 buffer (twice the L2 size)
  size_t flush_bytes = 0;
};

static std::string wigb_source(const std::vector<int>& classes, int warps, int precision, int xstage) {
  // Register caps, as the warps per SM each pass must allow (8-warp tiles run one
  // CTA per SM, 255 registers).  Measured on the 64-instance batch (B200, CUDA events):
  //   mixed x-pass 12 (168 registers, the same 72 B of spill as at 255): 253 -> 220 us
  //     against 8 warps per SM;
  //   mixed p-pass 12 (168 registers, ~1 KB of spill to L1-cached local memory; the
  //     1024-point FP64 Moyal pair holds 32 double2 per lane): 535 -> 487 us against 8;
  //   FP32 x-pass 16 (128 registers, no spill): 173 -> 164 us against 12;
  //   FP32 p-pass 12 (168 registers): 16 measured slower (347 -> 379 us).
  char head[512];
  const bool mixed = precision == WIGB_PREC_MIXED;
  const int xwps = mixed ? 12 : 16, pwps = 12;
  int xminb = warps == 8 ? 1 : std::max(1, xwps / warps), pminb = warps == 8 ? 1 : std::max(1, pwps / warps);
  // tuning override (read per compile): WIG_BATCH_WPS=x,p sets the x- and p-pass register
  // caps by the warps per SM they must allow (e.g. 12,8); 0 keeps the default
  if (const char* e = getenv("WIG_BATCH_WPS")) {
    int xw = 0, pw = 0;
    if (sscanf(e, "%d,%d", &xw, &pw) == 2) {
      if (xw > 0) xminb = std::max(1, xw / warps);
      if (pw > 0) pminb = std::max(1, pw / warps);
    }
  }
  // tuning override (read per compile): WIG_BATCH_NOINLINE=1 compiles each size class's
  // pass body as its own function
  const char* ni = getenv("WIG_BATCH_NOINLINE");
  const int noinline = ni && atoi(ni) ? 1 : 0;
  // failure-detection tests (read per compile): WIG_BATCH_TEST_STALL=1 builds the staged x-pass
  // with its row copies announced but never issued and a wait limit of 4096 polls, so a run
  // returns WIG_ERR_TIMEOUT quickly and leaves the context usable
  const char* ts = getenv("WIG_BATCH_TEST_STALL");
  const bool stall = ts && atoi(ts);
  // tuning override (read per compile): WIG_BATCH_DISS64=n runs the mixed form's dissipator in
  // FP64 on columns of at most n points (default 256; 0: FP32 dissipator on every size)
  int diss64 = 256;
  if (const char* dv = getenv("WIG_BATCH_DISS64")) {
    if (*dv) diss64 = std::max(0, atoi(dv));
  }
  snprintf(head, sizeof(head),
           "#define WIGB_WARPS %d\n#define WIGB_PREC %d\n#define WIGB_XMINB %d\n#define WIGB_PMINB %d\n"
           "#define WIGB_NOINLINE %d\n#define WIGB_XSTAGE %d\n#define WIGB_DISS64_MAXN %d\n#define WIGB_BULK 1\n"
           "%s#define WIGB_CASES(F)",
           warps, precision, xminb, pminb, noinline, xstage, diss64,
           stall ? "#define WIGB_TEST_STALL 1\n#define WIGB_WAIT_POLLS 4096L\n" : "");
  std::string src = head;
  for (int n : classes) src += " F(" + std::to_string(n) + ")";
  src += "\n";
  src += kJitBatchSource;
  return src;
}

extern "C" int wigb_jit_check(const int32_t* sizes, int64_t n_sizes, int32_t warps, int32_t precision, char* log,
                              int64_t log_cap) {
  if (!sizes || n_sizes < 1 || (warps != 2 && warps != 4 && warps != 8) ||
      (precision != WIGB_PREC_F32 && precision != WIGB_PREC_MIXED)) {
    fail(WIG_ERR_ARG, "wigb_jit_check: bad arguments");
    copy_log(g_last_error, log, log_cap);
    return WIG_ERR_ARG;
  }
  std::vector<int> cls(sizes, sizes + n_sizes);
  std::sort(cls.begin(), cls.end());
  cls.erase(std::unique(cls.begin(), cls.end()), cls.end());
  std::lock_guard<std::mutex> lk(g_mu);
  std::vector<char> cubin;
  std::string lg;
  int rc = nvrtc_compile(wigb_source(cls, warps, precision, batch_xstage(precision)), &cubin, &lg, true);
  copy_log(rc ? g_last_error : lg, log, log_cap);
  return rc;
}

static int wigb_compile(wigb_handle* h, int warps, BVariant* v) {
  const int xstage = batch_xstage(h->precision);
  const std::string src = wigb_source(h->classes, warps, h->precision, xstage);
  int smx = batch_smem_x(h->classes, warps, h->precision, xstage), smp = 0;
  for (int n : h->classes) smp = std::max(smp, batch_smem_p(n, warps));
  if (smx > 227 * 1024 || smp > 227 * 1024)
    return fail(WIG_ERR_ARG, "batched tile of %d warps needs %d / %d bytes of shared memory", warps, smx, smp);
  CUmodule mod;
  int rc = get_module(src, h->device, &mod);
  if (!rc) rc = get_fn(mod, "wigb_xpass", &v->fx, smx);
  if (!rc) rc = get_fn(mod, "wigb_ppass", &v->fp, smp);
  if (!rc) rc = get_fn(mod, "wigb_reduce", &v->fr, 0);
  if (!rc) rc = get_fn(mod, "wigb_scale", &v->fs, 0);
  if (rc) return rc;
  v->warps = warps;
  v->smem_x = smx;
  v->smem_p = smp;
  v->occ_x = occupancy(v->fx, warps * 32, smx);
  v->occ_p = occupancy(v->fp, warps * 32, smp);
  v->occ_x = std::max(v->occ_x, 1);
  v->occ_p = std::max(v->occ_p, 1);
  return WIG_OK;
}

// Work lists for a tile of `warps` warps: x-items of bx_rows(n_x, warps) rows,
// p-items of bp_cols(n_p, warps) columns; p-items of each instance contiguous
// (the last-CTA reduction reads them as a range), instances ordered by
// decreasing per-item cost so the persistent loop ends balanced.
static int wigb_set_warps(wigb_handle* h, int warps) {
  auto it = h->variants.find(warps);
  if (it == h->variants.end()) {
    BVariant v;
    if (int rc = wigb_compile(h, warps, &v)) return rc;
    it = h->variants.emplace(warps, v).first;
  }
  const BVariant& v = it->second;
  std::vector<int> order(h->count);
  for (int i = 0; i < h->count; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
    return (int64_t)h->binst[a].n_p * (h->binst[a].damp ? 4 : 1) > (int64_t)h->binst[b].n_p * (h->binst[b].damp ? 4 : 1);
  });
  std::vector<int2> xi, pi;
  for (int i : order) {
    wig::BInst& b = h->binst[i];
    const int rpb = wig::bx_rows(b.n_x, warps), cpb = wig::bp_cols(b.n_p, warps);
    if (b.n_p % rpb || b.n_x % cpb)
      return fail(WIG_ERR_ARG, "instance %d: grid %d x %d does not tile with %d warps", i, b.n_x, b.n_p, warps);
    b.xitem0 = (int)xi.size();
    b.n_xitems = b.n_p / rpb;
    for (int r = 0; r < b.n_p; r += rpb) xi.push_back(make_int2(i, r));
    b.pitem0 = (int)pi.size();
    b.n_pitems = b.n_x / cpb;
    for (int c = 0; c < b.n_x; c += cpb) pi.push_back(make_int2(i, c));
  }
  if (h->items_d) cudaFree(h->items_d);
  if (h->partials_d) cudaFree(h->partials_d);
  h->items_d = nullptr;
  h->partials_d = nullptr;
  WIG_CUDA(cudaMalloc(&h->items_d, (xi.size() + pi.size()) * sizeof(int2)));
  WIG_CUDA(cudaMemcpy(h->items_d, xi.data(), xi.size() * sizeof(int2), cudaMemcpyHostToDevice));
  WIG_CUDA(cudaMemcpy((int2*)h->items_d + xi.size(), pi.data(), pi.size() * sizeof(int2), cudaMemcpyHostToDevice));
  WIG_CUDA(cudaMalloc((void**)&h->partials_d, pi.size() * wig::NACC * sizeof(double)));
  WIG_CUDA(cudaMemcpy((void*)h->a.inst, h->binst.data(), h->binst.size() * sizeof(wig::BInst), cudaMemcpyHostToDevice));
  h->a.xitems = (const int2*)h->items_d;
  h->a.pitems = (const int2*)h->items_d + xi.size();
  h->a.partials = h->partials_d;
  h->n_xitems = (int)xi.size();
  h->n_pitems = (int)pi.size();
  h->grid_x = std::max(1, std::min(h->n_xitems, h->n_sm * v.occ_x));
  h->grid_p = std::max(1, std::min(h->n_pitems, h->n_sm * v.occ_p));
  h->warps = warps;
  if (h->gexec) { cudaGraphExecDestroy(h->gexec); h->gexec = nullptr; }
  return WIG_OK;
}

extern "C" int wigb_destroy(wigb_handle* h) {
  if (!h) return WIG_OK;
  cudaDeviceSynchronize();
  for (cudaEvent_t e : h->ev) cudaEventDestroy(e);
  if (h->gexec) cudaGraphExecDestroy(h->gexec);
  if (h->flush) cudaFree(h->flush);
  h->bufs.free_all();
  if (h->items_d) cudaFree(h->items_d);
  if (h->partials_d) cudaFree(h->partials_d);
  if (h->obs) cudaFree(h->obs);
  delete h;
  return WIG_OK;
}

extern "C" int wigb_create(const wigb_instance* inst, int64_t count, int32_t warps, int32_t precision,
                           wigb_handle** out) {
  if (!inst || !out || count < 1) return fail(WIG_ERR_ARG, "wigb_create: empty batch");
  *out = nullptr;
  if (precision != WIGB_PREC_F32 && precision != WIGB_PREC_MIXED)
    return fail(WIG_ERR_ARG, "wigb_create: precision must be WIGB_PREC_F32 or WIGB_PREC_MIXED");
  for (int64_t i = 0; i < count; ++i) {
    const wigb_instance& d = inst[i];
    if (d.n_x < 64 || d.n_x > 1024 || d.n_p < 64 || d.n_p > 1024 || (d.n_x & (d.n_x - 1)) || (d.n_p & (d.n_p - 1)))
      return fail(WIG_ERR_ARG, "instance %lld: grid %d x %d, batched grids must be powers of two in [64, 1024]",
                  (long long)i, d.n_x, d.n_p);
    if (!(d.x_amplitude > 0) || !(d.p_amplitude > 0) || !(d.hbar != 0) || !(d.mass != 0) || !std::isfinite(d.dt))
      return fail(WIG_ERR_ARG, "instance %lld: amplitudes > 0, hbar and mass nonzero, dt finite", (long long)i);
    if (d.damping_f != 0 && d.damping_f != 1)
      return fail(WIG_ERR_ARG, "instance %lld: damping_f must be 0 (|p|) or 1 (p^2/sqrt(p^2+eps))", (long long)i);
  }
  if (warps != 0 && warps != 2 && warps != 4 && warps != 8)
    return fail(WIG_ERR_ARG, "wigb_create: warps must be 0 (default 8), 2, 4 or 8");
  int device = 0;
  WIG_CUDA(cudaGetDevice(&device));
  WIG_CUDA(cudaFree(0));
  wigb_handle* h = new wigb_handle();
  h->device = device;
  h->count = (int)count;
  h->inst.assign(inst, inst + count);
  cudaDeviceGetAttribute(&h->n_sm, cudaDevAttrMultiProcessorCount, device);
  std::vector<int> cls;
  for (auto& d : h->inst) { cls.push_back(d.n_x); cls.push_back(d.n_p); }
  std::sort(cls.begin(), cls.end());
  cls.erase(std::unique(cls.begin(), cls.end()), cls.end());
  h->classes = cls;
  h->precision = precision;
  std::vector<float2> tw;
  std::vector<double2> tw64;
  std::map<int, int> tw_off;
  batch_twiddles(cls, &tw, &tw64, &tw_off);
  h->binst.resize(count);
  h->offsets.resize(count + 1);
  std::vector<float> ft;
  std::vector<double> fd;
  int64_t off = 0;
  for (int64_t i = 0; i < count; ++i) {
    const wigb_instance& d = h->inst[i];
    wig::BInst& b = h->binst[i];
    memset(&b, 0, sizeof(b));
    batch_instance_setup(d, b, &ft, &fd);
    b.off = off;
    h->offsets[i] = off;
    off += (int64_t)d.n_x * d.n_p;
    b.tw_x = tw_off[d.n_x];
    b.tw_p = tw_off[d.n_p];
  }
  h->total = off;
  h->offsets[count] = off;
  DevBuf& B = h->bufs;
  float2* tw_d = nullptr;
  double2* tw64_d = nullptr;
  float* ft_d = nullptr;
  double* fd_d = nullptr;
  wig::BInst* inst_d = nullptr;
  unsigned* cnt_d = nullptr;
  unsigned* tick_d = nullptr;
  unsigned* status_d = nullptr;
  double* scale_d = nullptr;
  int rc = B.alloc(&tw_d, tw.size(), tw.data());
  if (!rc) rc = B.alloc(&tw64_d, tw64.size(), tw64.data());
  if (!rc) rc = B.alloc(&ft_d, ft.size(), ft.data());
  if (!rc) rc = B.alloc(&fd_d, fd.size(), fd.data());
  if (!rc) rc = B.alloc(&inst_d, (size_t)count);
  if (!rc) rc = B.alloc(&cnt_d, (size_t)count);
  if (!rc) rc = B.alloc(&tick_d, (size_t)2);
  if (!rc) rc = B.alloc(&status_d, (size_t)1);
  if (!rc) rc = B.alloc(&scale_d, (size_t)count);
  if (!rc) {
    cudaError_t e = cudaMemset(cnt_d, 0, count * sizeof(unsigned));
    if (e == cudaSuccess) e = cudaMemset(tick_d, 0, 2 * sizeof(unsigned));
    if (e == cudaSuccess) e = cudaMemset(status_d, 0, sizeof(unsigned));
    if (e != cudaSuccess) rc = fail(WIG_ERR_CUDA, "cudaMemset: %s", cudaGetErrorString(e));
  }
  if (rc) { B.free_all(); delete h; return rc; }
  h->a.tw = tw_d;
  h->a.tw64 = tw64_d;
  h->a.ft = ft_d;
  h->a.fd = fd_d;
  h->a.inst = inst_d;
  h->a.counters = cnt_d;
  h->a.tickets = tick_d;
  h->a.status = status_d;
  h->a.scale = scale_d;
  if ((rc = wigb_set_warps(h, warps ? warps : 8))) { wigb_destroy(h); return rc; }
  *out = h;
  return WIG_OK;
}

extern "C" int wigb_offsets(wigb_handle* h, int64_t* offsets) {
  if (!h || !offsets) return fail(WIG_ERR_ARG, "wigb_offsets: null argument");
  for (int i = 0; i <= h->count; ++i) offsets[i] = h->offsets[i];
  return WIG_OK;
}

static int wigb_launch_run(wigb_handle* h, float* W, int64_t t_index0, int64_t n_prop, uint32_t flags,
                           cudaStream_t st) {
  const BVariant& v = h->variants[h->warps];
  wig::BArgs a = h->a;
  a.W = W;
  a.obs = h->obs;
  a.obs_stride = (int)(n_prop + 1);
  const int nt = v.warps * 32;
  int nxi = h->n_xitems, npi = h->n_pitems;
  {
    int mode = (flags & WIG_RUN_CONTINUE) ? 0 : 1, sample = 0;
    void* args[] = {&a, &npi, &mode, &sample};
    if (int rc = launch(v.fr, h->grid_p, nt, 0, st, args)) return rc;
  }
  const bool prof = (flags & WIG_RUN_PROFILE) && !(flags & WIG_RUN_GRAPH);
  if (prof) {
    while (h->ev.size() < 3 * (size_t)n_prop) {
      cudaEvent_t e;
      WIG_CUDA(cudaEventCreate(&e));
      h->ev.push_back(e);
    }
    h->ev_used = 3 * (size_t)n_prop;
  }
  const bool flush = prof && (flags & WIG_RUN_FLUSH_L2) && h->flush;
  for (int64_t n = 0; n < n_prop; ++n) {
    if (flush) WIG_CUDA(cudaMemsetAsync(h->flush, (int)(n & 0x7f), h->flush_bytes, st));
    if (prof) WIG_CUDA(cudaEventRecord(h->ev[3 * n], st));
    a.step = (unsigned)(t_index0 + n);   // the launch copies its parameters
    void* xargs[] = {&a, &nxi};
    if (int rc = launch(v.fx, h->grid_x, nt, v.smem_x, st, xargs)) return rc;
    if (prof) WIG_CUDA(cudaEventRecord(h->ev[3 * n + 1], st));
    int sample = (int)(n + 1);   // the polynomial potentials are time independent
    void* pargs[] = {&a, &npi, &sample};
    if (int rc = launch(v.fp, h->grid_p, nt, v.smem_p, st, pargs)) return rc;
    if (prof) WIG_CUDA(cudaEventRecord(h->ev[3 * n + 2], st));
  }
  void* sargs[] = {&a, &npi};
  return launch(v.fs, h->grid_p, nt, 0, st, sargs);
}

extern "C" int wigb_run(wigb_handle* h, void* W_dev, int64_t t_index0, int64_t n_prop, uint32_t flags,
                        double* obs_host, void* stream) {
  if (!h || !W_dev) return fail(WIG_ERR_ARG, "wigb_run: null handle or W");
  if (((uintptr_t)W_dev & 15) != 0) return fail(WIG_ERR_ARG, "wigb_run: W must be 16-byte aligned");
  if (n_prop < 0) return fail(WIG_ERR_ARG, "wigb_run: n_prop < 0");
  int cur;
  WIG_CUDA(cudaGetDevice(&cur));
  if (cur != h->device) return fail(WIG_ERR_ARG, "wigb_run: current device %d != handle device %d", cur, h->device);
  const size_t nobs = (size_t)h->count * (n_prop + 1) * WIG_NOBS;
  if (nobs > h->obs_cap) {
    if (h->gexec) { cudaGraphExecDestroy(h->gexec); h->gexec = nullptr; }
    if (int rc = ensure_obs(&h->obs, &h->obs_cap, nobs)) return rc;
  }
  cudaStream_t st = (cudaStream_t)stream;
  float* W = (float*)W_dev;
  if ((flags & WIG_RUN_FLUSH_L2) && (flags & WIG_RUN_PROFILE) && !(flags & WIG_RUN_GRAPH) && !h->flush) {
    int l2 = 0;
    cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, h->device);
    h->flush_bytes = 2 * (size_t)std::max(l2, 64 << 20);
    WIG_CUDA(cudaMalloc(&h->flush, h->flush_bytes));
  }
  if (flags & WIG_RUN_GRAPH) {
    const uint32_t key_flags = flags & ~(uint32_t)WIG_RUN_GRAPH;
    if (!(h->gexec && h->g_W == W_dev && h->g_t0 == t_index0 && h->g_n == n_prop && h->g_flags == key_flags &&
          h->g_warps == h->warps)) {
      if (h->gexec) { cudaGraphExecDestroy(h->gexec); h->gexec = nullptr; }
      cudaStream_t cap;
      WIG_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
      cudaGraph_t g;
      cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
      int rc = e == cudaSuccess ? wigb_launch_run(h, W, t_index0, n_prop, key_flags, cap)
                                : fail(WIG_ERR_CUDA, "cudaStreamBeginCapture: %s", cudaGetErrorString(e));
      cudaError_t e2 = cudaStreamEndCapture(cap, &g);
      cudaStreamDestroy(cap);
      if (rc) return rc;
      if (e2 != cudaSuccess) return fail(WIG_ERR_CUDA, "cudaStreamEndCapture: %s", cudaGetErrorString(e2));
      e = cudaGraphInstantiate(&h->gexec, g, 0);
      cudaGraphDestroy(g);
      if (e != cudaSuccess) { h->gexec = nullptr; return fail(WIG_ERR_CUDA, "cudaGraphInstantiate: %s", cudaGetErrorString(e)); }
      h->g_W = W_dev; h->g_t0 = t_index0; h->g_n = n_prop; h->g_flags = key_flags; h->g_warps = h->warps;
    }
    WIG_CUDA(cudaGraphLaunch(h->gexec, st));
  } else {
    if (int rc = wigb_launch_run(h, W, t_index0, n_prop, flags, st)) return rc;
  }
  if (obs_host) {
    unsigned status = 0;
    WIG_CUDA(cudaMemcpyAsync(obs_host, h->obs, nobs * sizeof(double), cudaMemcpyDeviceToHost, st));
    WIG_CUDA(cudaMemcpyAsync(&status, h->a.status, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    WIG_CUDA(cudaStreamSynchronize(st));
    if (status) {
      WIG_CUDA(cudaMemsetAsync(h->a.status, 0, sizeof(unsigned), st));
      return fail(WIG_ERR_TIMEOUT, "wigb_run: an x-pass wait for its staged rows gave up");
    }
    return check_finite(obs_host, nobs, "wigb_run observables");
  }
  return WIG_OK;
}

// Time each candidate tile shape on `probe_steps` steps of the batch (state in
// W_scratch, modified) and keep the fastest.
extern "C" int wigb_autotune(wigb_handle* h, void* W_scratch, int64_t probe_steps, int32_t* chosen, double* ms_out,
                             void* stream) {
  if (!h || !W_scratch || probe_steps < 1) return fail(WIG_ERR_ARG, "wigb_autotune: bad arguments");
  cudaStream_t st = (cudaStream_t)stream;
  const int cands[] = {8, 4, 2};
  int best = 0;
  double best_ms = 1e300;
  cudaEvent_t e0, e1;
  WIG_CUDA(cudaEventCreate(&e0));
  WIG_CUDA(cudaEventCreate(&e1));
  for (int ci = 0; ci < 3; ++ci) {
    const int w = cands[ci];
    if (wigb_set_warps(h, w) != WIG_OK) continue;   // e.g. a tile that does not fit: skip it
    if (int rc = wigb_run(h, W_scratch, 0, 1, 0, nullptr, stream)) return rc;   // warm-up
    WIG_CUDA(cudaEventRecord(e0, st));
    if (int rc = wigb_run(h, W_scratch, 0, probe_steps, WIG_RUN_CONTINUE, nullptr, stream)) return rc;
    WIG_CUDA(cudaEventRecord(e1, st));
    WIG_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    WIG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    if (ms_out) ms_out[ci] = ms;
    if (ms < best_ms) { best_ms = ms; best = w; }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (!best) return fail(WIG_ERR_ARG, "wigb_autotune: no tile shape fits this batch");
  if (int rc = wigb_set_warps(h, best)) return rc;
  if (chosen) *chosen = best;
  return WIG_OK;
}

extern "C" int wigb_profile(wigb_handle* h, double* ms_out, int64_t* launches) {
  if (!h || !ms_out) return fail(WIG_ERR_ARG, "wigb_profile: null argument");
  ms_out[0] = ms_out[1] = 0.;
  const size_t steps = h->ev_used / 3;
  for (size_t n = 0; n < steps; ++n) {
    float a = 0.f, b = 0.f;
    WIG_CUDA(cudaEventSynchronize(h->ev[3 * n + 2]));
    WIG_CUDA(cudaEventElapsedTime(&a, h->ev[3 * n], h->ev[3 * n + 1]));
    WIG_CUDA(cudaEventElapsedTime(&b, h->ev[3 * n + 1], h->ev[3 * n + 2]));
    ms_out[0] += a;
    ms_out[1] += b;
  }
  if (launches) *launches = (int64_t)steps;
  return WIG_OK;
}
