/*
 * wigner_b200.h -- C ABI of the B200 (sm_100a) Wigner2D / Dirac2D
 * split-operator propagators.
 *
 * The reference (cabrer7/PyWignerCUDA) drives its kernels from Python through
 * PyCUDA and a ctypes binding of cuFFT (cufft_wrapper.py:78-145).  This library
 * is the native layer under the Python drop-in classes
 * (pywignercuda_b200.GPU_Wigner2D_FFT / GPU_Wigner2D_ODM2 / GPU_Dirac2D): one
 * handle per propagator instance; expression strings are JIT-compiled by NVRTC
 * into the fused kernels the way the reference's SourceModule pastes them into
 * its kernel sources.
 *
 * Conventions
 *   - Plain C types only; device buffers are raw pointers owned by the caller
 *     (16-byte aligned, contiguous); scratch and tables are owned by the handle.
 *   - Every call returns an int status (WIG_OK or WIG_ERR_*); wig_last_error()
 *     gives the message of the calling thread's last failure.  No exception
 *     crosses the ABI.  (Replaces cufftCheckStatus, cufft_wrapper.py:67-75.)
 *   - One handle per stream; no internal host threads.
 *   - Grids: powers of two, Wigner n_x, n_p in [16, 4096], Dirac n_x, n_y in
 *     [16, 2048] (one fused pass holds a full line of the grid -- four spinor
 *     components for Dirac -- in shared memory).
 *   - Layout: (rows, cols) = (n_p, n_x) for Wigner, (n_y, n_x) per spinor
 *     component for Dirac, row-major, FFT-shifted (index 0 holds coordinate 0),
 *     complex128 interleaved -- the reference's layout
 *     (GPU_Wigner2D_FFT.py:577-581, GPU_Dirac2D.py:331-332).
 */
#ifndef WIGNER_B200_H
#define WIGNER_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define WIG_ABI_VERSION 4

enum wig_status {
  WIG_OK = 0,
  WIG_ERR_ARG = 1,         /* invalid descriptor / size / pointer            */
  WIG_ERR_NVRTC = 2,       /* expression strings failed to compile           */
  WIG_ERR_CUDA = 3,        /* CUDA runtime / driver error                    */
  WIG_ERR_TIMEOUT = 4,     /* a bounded device-side wait gave up             */
  WIG_ERR_NONFINITE = 5,   /* a recorded observable or norm became NaN / Inf */
  WIG_ERR_UNSUPPORTED = 6, /* valid request this build does not implement    */
  WIG_ERR_NOMEM = 7        /* device allocation failed                       */
};

enum wig_damping {
  WIG_DAMP_NONE = 0,
  WIG_DAMP_CALDEIRA_LEGGETT = 1, /* dampingFunction = 'CaldeiraLeggett' */
  WIG_DAMP_ODM = 2               /* dampingFunction = 'ODM'             */
};

enum wig_constants {
  WIG_CONST_CUDA_F = 0, /* kernel constants rounded by '%f' as the reference does */
  WIG_CONST_EXACT = 1   /* full double precision                                 */
};

enum wig_precision { WIG_PREC_C128 = 0, WIG_PREC_F32 = 1 };

enum wig_splitting {
  WIG_SPLIT_LIE = 0,       /* kinetic then potential (GPU_Wigner2D_FFT.Run :1884-1913)           */
  WIG_SPLIT_STRANG_GP = 1  /* half potential, kinetic, half potential, each half with the
                              Gross-Pitaevskii term when gp_coefficient != 0; observables after
                              every step (GPU_Wigner2D_GPitaevskii.Run, GPU_Wigner2D_GPitaevskii.py
                              :1897-1990)                                                         */
};

enum wig_potential_phase {
  WIG_PHASE_MOYAL = 0, /* exp(-i dt [V(x - hbar theta/2) - V(x + hbar theta/2)] / hbar)
                          (expPotential_source, GPU_Wigner2D_FFT.py:80-126)            */
  WIG_PHASE_KVN = 1    /* classical Liouville (KvN) factor exp(+i dt V'(t, x) theta) from the
                          dpotential string (exp_PotentialKvN_source :27-75,
                          GPU_FokkerPlank2D_FFT :2242-2459)                          */
};

/* wig_run / dirac_run flags */
#define WIG_RUN_CONTINUE 1u /* W continues an earlier call: skip the entry normalisation */
#define WIG_RUN_PROFILE 2u  /* time every x-pass / p-pass launch with CUDA events (wig_profile) */
#define WIG_RUN_GRAPH 4u    /* wigb_run: capture the launch sequence in a CUDA graph once, replay it */
#define WIG_RUN_FLUSH_L2 8u /* wigb_run with WIG_RUN_PROFILE (no graph): before every step, write a
                               buffer twice the L2 size, outside the timed launches, so each step
                               starts from a cold L2 */

#define WIG_NOBS 11   /* norm, <x>, <x^2>, <p>, <p^2>, <xp>, <V'>, <pV'>, <xV'>, <H>, negative area */
#define DIRAC_NOBS 10 /* <x>, <y>, <alpha1>, <alpha2>, <beta>, <K>, <A0>, <px>, <py>, norm_kept */
#define DIRAC3_NOBS 12 /* <x>, <y>, <z>, <alpha1>, <alpha2>, <alpha3>, <A0>, <px>, <py>, <pz>, <K>, norm */

typedef struct wig_handle wig_handle;
typedef struct dirac_handle dirac_handle;

/* Wigner2D instance description: the constructor arguments of
 * GPU_Wigner2D_FFT / GPU_Wigner2D_ODM2 (GPU_Wigner2D_FFT.py:1718-1720,1981-1984)
 * plus the attributes an instance sets before construction. */
typedef struct wig_desc {
  int32_t abi_version;         /* WIG_ABI_VERSION                                   */
  int32_t n_x, n_p;            /* X_gridDIM, P_gridDIM                              */
  int32_t damping;             /* wig_damping; used only when gamma != 0 (Run :1901) */
  int32_t kinetic_from_string; /* 0: p*lambda/mass phase (GPU_Wigner2D_FFT.Run)
                                  1: kinetic string phase (GPU_Wigner2D_ODM2.Run)    */
  int32_t constants;           /* wig_constants                                     */
  int32_t precision;           /* wig_precision                                     */
  int32_t n_lindblad;          /* ODM: 1 (GPU_Wigner2D_FFT) or 2 (GPU_Wigner2D_ODM2)  */
  int32_t potential_phase;     /* wig_potential_phase (KvN: damping none or Caldeira-Leggett) */
  int32_t skip_normalise;      /* 1: damped steps are not renormalised (GPU_FokkerPlank2D_FFT
                                  with normalization != 'Wigner', :2404-2406)           */
  int32_t splitting;           /* wig_splitting (Strang: Moyal phase only)              */
  int32_t reserved0;
  double x_amplitude, p_amplitude;
  double hbar, mass, dt;
  double d_theta, d_lambda, gamma;
  double epsilon, l_material;  /* ODM (SetA_ODM :1206)                              */
  double weight1, weight2;     /* ODM2 Lindblad weights (:2169-2176)                 */
  double gp_coefficient;       /* GPitaevskiiCoeff a_GP (WIG_SPLIT_STRANG_GP)          */
  const char* potential;       /* potentialString, C expression in (t, x)           */
  const char* kinetic;         /* kinematicString, C expression in p                */
  const char* fp_damping;      /* fp_Damping_String, C expression in p              */
  const char* dpotential;      /* dPotentialString, C expression in (t, x); used by
                                  WIG_PHASE_KVN (NULL -> "0.")                          */
  /* Exact host tables of the observables (Run :1785-1792, :1747); NULL -> built
   * by the library (shifted linspace grids; zeros for dV / V0). */
  const double* x_table;       /* [n_x] */
  const double* p_table;       /* [n_p] */
  const double* theta_table;   /* [n_p] */
  const double* lambda_table;  /* [n_x] */
  const double* dv_table;      /* [n_x] dPotential(0, x) */
  const double* v0_table;      /* [n_x] Potential(0, x)  */
  /* Values of cf[0] .. cf[7], which the expression strings may use: instances
   * that differ only in these share one compiled module. */
  double coef[8];
} wig_desc;

/* Replaces GPU_Wigner2D_FFT.__init__ (:1718-1751): SetPhaseSpaceBox2D,
 * SetCUDA_Constants (:833-842), SetFFT_Plans (:859-865), SetCUDA_Functions
 * (:869-906, NVRTC instead of SourceModule). */
int wig_create(const wig_desc* desc, wig_handle** out);

/* The hot loop of GPU_Wigner2D_FFT.Run / GPU_Wigner2D_ODM2.Run (:1843-1914):
 * normalises W (as Run does on entry, :1779-1780), then performs n_prop
 * propagations starting at time index t_index0 (t = t_index * dt), in place on
 * the device array W ((n_p, n_x) complex128).  flags & WIG_RUN_CONTINUE: W is
 * the state an earlier call returned; no entry normalisation.  obs_host (may be NULL) receives
 * (n_prop + 1) x WIG_NOBS doubles: sample k is taken before propagation k, the
 * last one after the final propagation.  Run(timeSteps) == n_prop = timeSteps+1
 * keeping the first timeSteps+1 samples.  stream: a cudaStream_t (NULL = legacy
 * default stream).  Returns after the stream is synchronised when obs_host is
 * given, otherwise asynchronously. */
int wig_run(wig_handle* h, void* W_dev, int64_t t_index0, int64_t n_prop, uint32_t flags,
            double* obs_host, void* stream);

/* wig_run on host buffers: W_in (host, complex128) is copied to the device,
 * propagated, and copied back into W_out (host, may alias W_in); the run's
 * device buffer is owned by the handle.  (Run's W_init upload :1778 and W_end
 * download :1954.) Synchronous. */
int wig_run_host(wig_handle* h, const void* W_in_host, void* W_out_host, int64_t t_index0,
                 int64_t n_prop, uint32_t flags, double* obs_host, void* stream);

/* wig_run over `count` independent instances (each with its own handle and W)
 * stepped in lock-step on one stream: step k of every instance is launched
 * before step k+1 of any.  obs_host may be NULL or hold per-instance pointers
 * (NULL entries allowed).  The reference runs one instance per Run()
 * (GPU_Wigner2D_FFT.py:1843); this batches that loop. */
int wig_run_many(wig_handle* const* handles, void* const* W_dev, int64_t count, int64_t t_index0,
                 int64_t n_prop, uint32_t flags, double* const* obs_host, void* stream);

/* Per-kernel device time of the handle's last run made with WIG_RUN_PROFILE:
 * ms_out[0] = summed x-pass milliseconds, ms_out[1] = summed p-pass
 * milliseconds, *launches = launches of each.  Synchronises on the events.
 * (No counterpart in the reference, which times whole runs with %time.) */
int wig_profile(wig_handle* h, double* ms_out, int64_t* launches);

/* Replaces the cufftDestroy calls at the end of Run (:1960-1962). */
int wig_destroy(wig_handle* h);

/* Dirac2D instance: GPU_Dirac2D(gridDIM, amplitude, dt, ...) and the attributes
 * mass, c, hBar, Potential_{0..3}_String (GPU_Dirac2D.py:306,356-380). */
typedef struct dirac_desc {
  int32_t abi_version;
  int32_t n_x, n_y;
  int32_t constants;           /* wig_constants */
  int32_t precision;           /* wig_precision */
  int32_t reserved;
  double x_amplitude, y_amplitude;
  double mass, c, hbar, dt;
  const char* a0;              /* Potential_0_String, C expression in (t, x, y) */
  const char* a1;
  const char* a2;
  const char* a3;
  const double* x_table;       /* [n_x] shifted X  (NULL -> built) */
  const double* y_table;       /* [n_y] shifted Y  */
  const double* px_table;      /* [n_x] shifted Px */
  const double* py_table;      /* [n_y] shifted Py */
  double coef[8];              /* values of cf[0] .. cf[7] in the expressions */
} dirac_desc;

/* Replaces GPU_Dirac2D.__init__ (GPU_Dirac2D.py:306-392). */
int dirac_create(const dirac_desc* desc, dirac_handle** out);

/* GPU_Dirac2D.Run's loop (:1040-1111): n_steps >= 1 propagations at
 * t = (t_index0 + k) * dt, k = 1..n_steps, in place on the device spinor psi
 * ((4, n_y, n_x) complex128), which holds the normalised final spinor on
 * return (Normalize_X, :1103).  obs_host (may be NULL) receives
 * n_steps x DIRAC_NOBS doubles, sample k taken before propagation k + 1, as
 * Run records them. */
int dirac_run(dirac_handle* h, void* psi_dev, int64_t t_index0, int64_t n_steps,
              double* obs_host, void* stream);

/* dirac_run over `count` independent instances stepped in lock-step on one
 * stream (the Dirac counterpart of wig_run_many). */
int dirac_run_many(dirac_handle* const* handles, void* const* psi_dev, int64_t count, int64_t t_index0,
                   int64_t n_steps, double* const* obs_host, void* stream);

/* dirac_run on host buffers (Psi_init upload :1002-1005, Psi_end download :1119). */
int dirac_run_host(dirac_handle* h, const void* psi_in_host, void* psi_out_host, int64_t t_index0,
                   int64_t n_steps, double* obs_host, void* stream);

int dirac_destroy(dirac_handle* h);

/* Dirac3D instance: GPU_Dirac3D(gridDIM, amplitude, dt, ...) and the attributes
 * mass, c, hBar, Potential_{0..3}_String (GPU_Dirac3D.py:616-757).  Grids are
 * powers of two in [16, 512] per axis; the spinor is (4, n_z, n_y, n_x)
 * complex128, each axis FFT-shifted. */
typedef struct dirac3_handle dirac3_handle;
typedef struct dirac3_desc {
  int32_t abi_version;
  int32_t n_x, n_y, n_z;
  int32_t constants;           /* wig_constants */
  int32_t precision;           /* wig_precision (WIG_PREC_C128) */
  double x_amplitude, y_amplitude, z_amplitude;
  double mass, c, hbar, dt;    /* mass > 0 */
  const char* a0;              /* Potential_0_String, C expression in (t, x, y, z) */
  const char* a1;
  const char* a2;
  const char* a3;
  double coef[8];              /* values of cf[0] .. cf[7] in the expressions */
} dirac3_desc;

/* Replaces GPU_Dirac3D.__init__'s kernel compilation and plan (GPU_Dirac3D.py:690-757). */
int dirac3_create(const dirac3_desc* desc, dirac3_handle** out);

/* GPU_Dirac3D.Run's loop (:1325-1465): n_steps >= 1 propagations at
 * t = (t_index0 + k) * dt, k = 1..n_steps, in place on the device spinor psi.
 * Without WIG_RUN_CONTINUE the spinor is first normalised (Normalize_GPU,
 * :1323) and the momentum-space norm of the t_index = 1 spectrum is taken
 * again; with it, the run continues an earlier one on this handle.  obs_host
 * (may be NULL) receives n_steps x DIRAC3_NOBS doubles, sample k taken before
 * propagation k + 1 as Run records them (the momentum averages divided by the
 * step-1 norm, Compute_Ehrenfest_P :1366-1395, always computed).  Synchronous
 * when obs_host is given. */
int dirac3_run(dirac3_handle* h, void* psi_dev, int64_t t_index0, int64_t n_steps, uint32_t flags,
               double* obs_host, void* stream);

/* dirac3_run on host buffers (the Psi_init upload :1296-1299, Psi_end download :1474). */
int dirac3_run_host(dirac3_handle* h, const void* psi_in_host, void* psi_out_host, int64_t t_index0,
                    int64_t n_steps, uint32_t flags, double* obs_host, void* stream);

int dirac3_destroy(dirac3_handle* h);

/* Compile-only check of a Dirac3D instance's kernels (no GPU needed). */
int dirac3_jit_check(const dirac3_desc* desc, char* log, int64_t log_cap);

/* ---------------------------------------------------------------- batched form
 * Many independent Wigner2D instances with polynomial potentials
 * V(x) = v4 x^4 + v2 x^2 + v1 x + v0, kinetic p^2/2m, Caldeira-Leggett damping
 * (gamma != 0) with f(p) = |p| or p^2/sqrt(p^2 + f_eps), on uneven grids
 * (powers of two in [64, 1024]), advanced together.  The state is real FP32
 * storage, one float per grid point: W is a Wigner function, so two real rows
 * (x-pass) or columns (p-pass) share each complex transform, and the
 * imaginary rounding noise of a complex step is not kept.  Precision of the
 * arithmetic, one per batch:
 *   WIGB_PREC_F32    FP32 transforms and factors throughout;
 *   WIGB_PREC_MIXED  the kinetic and Moyal transform pairs and their factors
 *                    in FP64 (and the dissipator pairs, up to 256-point
 *                    columns; FP32 above), each FP64 result rounded to the
 *                    FP32 state stochastically: a function of the inputs and
 *                    the step index t_index0 + n, so a run is reproducible
 *                    (pass t_index0 on a continued run for fresh rounding).
 * Both form the phase arguments in FP64 and reduce them to one turn, and keep
 * the observables in FP64 (per-column moments, compensated per-instance sums).
 * Constants are exact (no '%f' rounding).  No counterpart in the reference,
 * which runs one complex128 instance per Run() (GPU_Wigner2D_FFT.py:1843); the
 * step is the same Lie split (:1884-1913). */
#define WIGB_PREC_F32 0
#define WIGB_PREC_MIXED 1

typedef struct wigb_instance {
  int32_t n_x, n_p;
  int32_t damping_f;  /* 0: f = |p|, 1: f = p^2/sqrt(p^2 + f_eps) */
  int32_t reserved;
  double x_amplitude, p_amplitude, hbar, mass, dt;
  double d_theta, d_lambda, gamma, f_eps;
  double v4, v2, v1, v0;
} wigb_instance;

typedef struct wigb_handle wigb_handle;

/* warps: tile shape (warps per CTA, 2 / 4 / 8; 0 = 8 until wigb_autotune picks one).
 * precision: WIGB_PREC_F32 or WIGB_PREC_MIXED. */
int wigb_create(const wigb_instance* instances, int64_t count, int32_t warps, int32_t precision,
                wigb_handle** out);

/* offsets[count + 1]: element offset of each instance's (n_p, n_x) float
 * block in the packed state buffer; offsets[count] = total elements. */
int wigb_offsets(wigb_handle* h, int64_t* offsets);

/* Normalise (unless flags & WIG_RUN_CONTINUE) and advance every instance of
 * the packed real FP32 state W (16-byte aligned) by n_prop propagations (t = t_index * dt).
 * obs_host (may be NULL): count x (n_prop + 1) x WIG_NOBS doubles, instance
 * major; with it the call synchronises the stream and returns WIG_ERR_TIMEOUT
 * (a bounded device-side wait gave up) or WIG_ERR_NONFINITE before returning
 * numbers.  Without it the call is asynchronous and those checks wait for the
 * next call that asks for observables (the timeout flag persists until read).
 * flags & WIG_RUN_GRAPH: the launch sequence is captured into a CUDA
 * graph on first use (per W, t_index0, n_prop, flags, tile shape) and replayed. */
int wigb_run(wigb_handle* h, void* W_dev, int64_t t_index0, int64_t n_prop, uint32_t flags,
             double* obs_host, void* stream);

/* The project's autotuner: times each candidate tile shape (8, 4, 2 warps per
 * CTA) on probe_steps steps of the batch using W_scratch (overwritten) and
 * keeps the fastest; *chosen gets it, ms_out[3] the timings (0 if skipped). */
int wigb_autotune(wigb_handle* h, void* W_scratch, int64_t probe_steps, int32_t* chosen,
                  double* ms_out, void* stream);

/* Per-pass device time of the last wigb_run made with WIG_RUN_PROFILE and
 * without WIG_RUN_GRAPH: ms_out[0] x-pass, ms_out[1] p-pass (summed). */
int wigb_profile(wigb_handle* h, double* ms_out, int64_t* launches);

int wigb_destroy(wigb_handle* h);

/* Compile-only check (no GPU) of the batched kernels for the given grid sizes,
 * tile shape and precision; log receives the NVRTC / ptxas report. */
int wigb_jit_check(const int32_t* sizes, int64_t n_sizes, int32_t warps, int32_t precision, char* log,
                   int64_t log_cap);

/* ---- Adjoint (differentiable) form.  No counterpart in the reference, which
 * has no gradients.  One Wigner2D grid (powers of two in [64, 1024] per axis)
 * advanced by the Lie step of GPU_Wigner2D_FFT.Run (:1884-1913)
 *   W_{n+1} = N(C P(eps_n) K W_n),
 * K the kinetic x-pass (p^2/2m, r_lambda), P the Moyal p-pass with
 * V(x) = v4 x^4 + v2 x^2 + v0 + eps_n x, r_theta and the absorbing masks;
 * eps_n is a control per step read from device memory.  With gamma != 0, C is
 * the Caldeira-Leggett order-3 step (:1145-1157, f(p) = |p| when f_eps = 0,
 * else p^2/sqrt(p^2 + f_eps)) and N the normalisation U -> U / (dX dP sum U)
 * (:1912-1913); with gamma = 0 both are the identity.  State: (n_p, n_x)
 * FFT-shifted, device, complex64 (WIGA_PREC_C64: FP32 transforms) or
 * complex128 (WIGA_PREC_C128: FP64 transforms). */
#define WIGA_PREC_C64 0
#define WIGA_PREC_C128 1
typedef struct wiga_desc {
  int32_t abi_version;   /* WIG_ABI_VERSION */
  int32_t n_x, n_p;
  int32_t precision;     /* WIGA_PREC_C64 or WIGA_PREC_C128 */
  double x_amplitude, p_amplitude, hbar, mass, dt, d_theta, d_lambda;
  double v4, v2, v0;
  double gamma, f_eps;
} wiga_desc;

typedef struct wiga_handle wiga_handle;

int wiga_create(const wiga_desc* desc, wiga_handle** out);

/* Replace the potential coefficients of the handle (the next forward and
 * adjoint steps use them). */
int wiga_set_potential(wiga_handle* h, double v4, double v2, double v0);

/* n_steps forward steps from step index step0, W in place (normalised on
 * return when damped).  eps_dev: device double array indexed by step
 * (>= step0 + n_steps entries).  Optional (may be NULL) records of each step,
 * the inputs wig_step_adjoint needs: Y_dev [n_steps][n_p][n_x] receives
 * Y_n = K W_n; U_dev [n_steps][n_p][n_x] the damped step's output before
 * normalisation; s_dev (device double2, indexed by step) its sum dX dP sum U.
 * Asynchronous on `stream`. */
int wiga_forward(wiga_handle* h, void* W_dev, const double* eps_dev, int64_t step0, int64_t n_steps,
                 void* Y_dev, void* U_dev, void* s_dev, void* stream);

/* One adjoint step n.  On entry lam_dev (device, the state's type) holds
 * dL/dW_{n+1}, on exit dL/dW_n = K^H P(eps_n)^H C^H N_n^H dL/dW_{n+1}
 * (gradients in the convention dL = Re sum conj(grad) dW, the one torch uses
 * for complex tensors).  Y_dev: Y_n; damped: U_dev = U_n and s_dev (indexed by
 * step) from wiga_forward (NULL when undamped).  grad_dev (device double,
 * [steps][3]) receives at [3 step .. 3 step + 2] dL/d eps_n and step n's
 * shares of dL/dv4 and dL/dv2 (dL/dv4 is their sum over the steps).
 * Asynchronous on `stream`. */
int wig_step_adjoint(wiga_handle* h, void* lam_dev, const void* Y_dev, const void* U_dev, const void* s_dev,
                     const double* eps_dev, int64_t step, double* grad_dev, void* stream);

/* The adjoint steps step0 + n_steps - 1 down to step0 in one call (the same
 * launches as n_steps calls of wig_step_adjoint, with the arguments checked once):
 * Y_dev and (damped) U_dev are that segment's records from wiga_forward
 * ([n_steps][n_p][n_x], record k for step step0 + k).  No counterpart in the
 * reference (it has no gradients).  Asynchronous on `stream`. */
int wiga_adjoint_sweep(wiga_handle* h, void* lam_dev, const void* Y_dev, const void* U_dev, const void* s_dev,
                       const double* eps_dev, int64_t step0, int64_t n_steps, double* grad_dev, void* stream);

int wiga_destroy(wiga_handle* h);

/* Compile-only check (no GPU) of the adjoint kernels for the descriptor's grid. */
int wiga_jit_check(const wiga_desc* desc, char* log, int64_t log_cap);

/* WIG_SPLIT_STRANG_GP with gp_coefficient != 0: the per-step sum_x P(x)^2 dx of
 * the x-marginal P after each kinetic step of the last wig_run on this handle
 * (GPU_Wigner2D_GPitaevskii ProbabilitySquare_average, :1951); n <= that run's
 * n_prop values into out (host).  Synchronises the handle's last stream. */
int wig_run_probability_square(wig_handle* h, double* out, int64_t n);

/* ---- Imaginary-time (Bloch) steps of GPU_Wigner2D_GPitaevskii_Bloch
 * (GPU_Wigner2D_GPitaevskii.py:2064-2545) on a WIG_SPLIT_STRANG_GP handle.
 * stats[WIG_BLOCH_NSTATS]: <x>, <x^2>, <p>, <p^2>, <K(p) + V(0, x)> (K from the
 * kinetic string, as the class's Hamiltonian), purity Re / Im
 * (2 pi hbar dXdP sum W^2, Purity_GPU :1738-1741), the mean-field energy
 * 0.5 a_GP sum_x P(x)^2 dx (NonLinearEnergy :1757-1758), 1 if some
 * p-marginal value is negative (computed when W0 != NULL), the norm used. */
#define WIG_BLOCH_NSTATS 10

/* stats of W (complex128 (n_p, n_x), device); normalise != 0 first divides W by
 * (sum W dX) dP as Run does with its initial state (:2129-2131).  Synchronous. */
int wig_bloch_stats(wig_handle* h, void* W_dev, int32_t normalise, double* stats, void* stream);

/* One imaginary-time step of size dtb at t = t_index dt, in place: [mean-field
 * exponent] half potential (Kernel_Bloch, exp(-dtb/4 [V(x - hbar theta/2) +
 * V(x + hbar theta/2)])) -> kinetic (exp(-dtb/2 [K(p + hbar lambda/2) +
 * K(p - hbar lambda/2)])) -> [mean-field exponent] half potential; then, when
 * W0 != NULL (Run_ExitedState1), W -= (2 pi hbar dXdP sum W W0) W0; then
 * W /= sum W (dX dP); stats of the result.  The caller keeps the reference's
 * accept / reject logic (energy must fall, |purity| < 1, and for the excited
 * state no negative p-marginal; otherwise halve dtb and restore W).
 * Synchronous. */
int wig_bloch_step(wig_handle* h, void* W_dev, int64_t t_index, double dtb, const void* W0_dev, double* stats,
                   void* stream);

/* Compile-only check of an instance's kernels: builds the JIT source the way
 * wig_create / dirac_create do and compiles it with NVRTC for sm_100a without
 * loading it (no GPU needed).  log (may be NULL) receives the NVRTC log with
 * the ptxas register / spill report, or the error.  The compile step of the
 * reference's SourceModule calls (GPU_Wigner2D_FFT.py:869-906,
 * GPU_Dirac2D.py:369-388). */
int wig_jit_check(const wig_desc* desc, char* log, int64_t log_cap);
int dirac_jit_check(const dirac_desc* desc, char* log, int64_t log_cap);

/* The observables of a Wigner function W ((n_p, n_x) complex128, device) --
 * the 11 values wig_run records for a sample it does not renormalise (norm,
 * <x>, <x^2>, <p>, <p^2>, <xp>, <V'>, <pV'>, <xV'>, <H>, negative area) --
 * written to obs_dev[WIG_NOBS] (device), for callers that cannot allocate
 * device memory (an allocator hook, where cudaMalloc would re-enter the
 * allocator; a deployment that forbids allocation after start-up).  Host
 * functions run by cudaLaunchHostFunc may not call it: CUDA forbids every
 * CUDA call there.
 * No counterpart in the reference.  It allocates nothing: its per-row partial
 * sums live in a fixed device array of 4096 rows x 12 doubles (384 KB per
 * device, held until the process exits), so n_p <= 4096 and n_x <= 4096,
 * larger grids are rejected with WIG_ERR_ARG.  The tables (x, p, dV/dx,
 * V(0, x); the library's shifted grids) are device arrays the caller owns;
 * dx, dp are the grid steps and mass enters <H> = <p^2/2m + V>.  All calls on
 * a device share the array and each overwrites the rows it reads, so calls
 * whose kernels overlap on the GPU race.  The first call on a device looks up
 * the array's address with that device current: make it before any stream
 * capture.  Under lazy module loading (CUDA's default) that first call also
 * loads the module that holds the array, an allocation by the driver: make it
 * at start-up (a warm-up call), before allocation is forbidden.  Asynchronous
 * on `stream`. */
int wig_observables_noalloc(const void* W_dev, int32_t n_x, int32_t n_p, double dx, double dp, double mass,
                            const double* x_tab_dev, const double* p_tab_dev, const double* dv_tab_dev,
                            const double* v0_tab_dev, double* obs_dev, void* stream);

/* Message of the calling thread's last failed call ("" if none). */
const char* wig_last_error(void);

/* WIG_ABI_VERSION of the loaded library. */
int wig_abi_version(void);

#ifdef __cplusplus
}
#endif

#endif /* WIGNER_B200_H */
