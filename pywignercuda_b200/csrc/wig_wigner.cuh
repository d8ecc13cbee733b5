// Wigner2D split-operator step for sm_100a: two fused passes per step.
//
// Layout: W is (N_p, N_x) complex128, row-major, x contiguous, FFT-shifted in
// both axes (array index 0 holds coordinate 0) -- the reference's layout
// (GPU_Wigner2D_FFT.py:577-581).
//
//  x-pass (one CTA = ROWS contiguous rows):
//      prologue: deferred normalisation W <- W * s, s = 1/(dX dP sum W) taken
//                from the previous pass's per-CTA partial sums;
//      row FFT x->lambda, kinetic factor, row IFFT (1/N_x folded in).
//      (expPLambda_source :131-158 / expPLambdaKinetic_source :162-200 between
//       Fourier_X_To_Lambda_GPU and Fourier_Lambda_To_X_GPU, :1885-1888)
//  p-pass (one CTA = a tile of C columns x all N_p rows):
//      column FFT p->theta, Moyal potential factor, diffusion factor and the
//      two absorbing masks, column IFFT (1/N_p folded in)
//      (expPotential_source :80-126, :1891-1899);
//      Caldeira-Leggett order 3 (CaldeiraDissipatorOrder3 :1145-1157) on the
//      tile still in shared memory;
//      epilogue: store W' and this CTA's partial sums of the 10 observables
//      plus sum W (Run :1857-1878,1912).
//
// Each pass reads and writes W once (64 B per grid point per step).
#pragma once
#include "wig_fft.cuh"

// largest Stockham radix of the complex128 x-pass / p-pass transforms (the JIT sets them)
#ifndef WIG_XR
#define WIG_XR 8
#endif
#ifndef WIG_PR
#define WIG_PR 8
#endif

namespace wig {

constexpr int NACC = 12;   // sumRe, sumIm, x, x^2, p, p^2, xp, V', pV', xV', H, negative
constexpr int NOBS = 11;   // norm, x, x^2, p, p^2, xp, V', pV', xV', H, negative area
constexpr int NIM = 10;    // imaginary parts of the sums of observables 1..10

struct WigArgs {
  // kernel constants exactly as the reference's kernels see them
  // (SetCUDA_Constants :833-842: '%f'-rounded unless exact mode is asked for)
  double dt, dx, dp, dtheta, dlambda, mass, hbar, D_theta, D_lambda;
  // host-side exact values (the reference's observable tables and sums)
  double dX, dP, mass_exact;
  // Caldeira-Leggett polynomial W + c3 D(W + c12 D(W + c1 D W)) (Horner form of
  // W + a(1 + a/2)(1 + a/3)W, a = 2 i gamma dt D)
  double2 cl_k1, cl_k12, cl_c3;
  // 1-D device tables
  const double* x_tab;     // [n_x] shifted X (exact)
  const double* p_tab;     // [n_p] shifted P (exact)
  const double* dV_tab;    // [n_x] dPotential(0, x)
  const double* V0_tab;    // [n_x] Potential(0, x)
  const double* theta_s;   // [n_p] exact shifted Theta / n_p
  const double* r_lambda;  // [n_x] exp(-D_Lambda lambda^2)       (per frequency)
  const double* r_theta;   // [n_p] exp(-D_Theta theta^2 dt)      (per frequency)
  const double* mask1;     // [n_x] 1 - exp(-(x - x_max)^2/(10 dx)^2)
  const double* mask2s;    // [n_x] (1 - exp(-(x + x_max)^2/(10 dx)^2)) / n_p
  const double* sfp;       // [n_p] sign(p) f(p)   (theta_fp_source :399-431)
  const double2* tw_x;     // [n_x] exp(-2 pi i m / n_x)
  const double2* tw_p;     // [n_p]
  double* partials;        // [n_cta][NACC]
  // [n_cta][NIM] imaginary parts of the moment sums, written with `partials` by the passes of
  // plans whose steps do not keep sum W real (ODM damping); null otherwise
  double* partials_im;
  int n_partials;          // CTAs that wrote `partials`
  // ODM Lindblad damping (SetA_ODM :1206-1244, _Lindbladian_ODM :1516-1634), exact host values
  const double* lambda_tab; // [n_x] exact shifted Lambda
  double hbar_exact, L_material;
  // Strang splitting / Gross-Pitaevskii (GPU_Wigner2D_GPitaevskii)
  const double* r_theta_half;  // [n_p] exp(-0.5 D_Theta theta^2 dt)  (expPotential_source :66)
  double gp_coef;              // a_GP as the kernels see it
  double coef[8];           // cf[0..7] of the expression strings
  // register-FFT twiddle tables (wig_rfft.cuh layout, 2 n entries) of the
  // register-FFT passes (wig_wigner_rf.cuh); null when the plan uses the Stockham ones
  const double2* rtw_x;
  const double2* rtw_p;
  int* status;              // [1] set to 1 by a bounded wait that gave up (read and cleared by the host)
};

// ------------------------------------------------------------------ reductions
template <int NT, int NV>
__device__ __forceinline__ void block_sum(double (&acc)[NV], double (*red)[NV]) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    double x = acc[v];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    acc[v] = x;
  }
  if (lane == 0) {
#pragma unroll
    for (int v = 0; v < NV; ++v) red[warp][v] = acc[v];
  }
  __syncthreads();
  if (threadIdx.x < NV) {
    double s = 0.;
    for (int w = 0; w < NT / 32; ++w) s += red[w][threadIdx.x];
    red[0][threadIdx.x] = s;     // only lane threadIdx.x < NV reads/writes column threadIdx.x
  }
  __syncthreads();
}

// numpy's complex reciprocal 1/(a + i b) (Smith's method)
__device__ __forceinline__ double2 crecip(double2 z) {
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

// Scale modes: 0 = none; 1 = the initial normalisation of Run (:1779-1780,
// norm = (sum W * dX) * dP); 2 = the per-step one (:1912-1913,
// norm = sum W * (dX * dP)).  Reduces the previous pass's partials, returns
// s = 1/norm (or 1) and, when obs_row != nullptr, writes that sample's 11
// observables.
template <int NT>
__device__ __forceinline__ double2 consume_partials(const WigArgs& a, int mode, double* obs_row,
                                                    double (*red)[NACC]) {
  double acc[NACC];
#pragma unroll
  for (int v = 0; v < NACC; ++v) acc[v] = 0.;
  const int ncol = obs_row ? NACC : 2;
  for (int i = threadIdx.x; i < a.n_partials; i += NT) {
    const double* p = a.partials + (size_t)i * NACC;
#pragma unroll
    for (int v = 0; v < NACC; ++v)
      if (v < ncol) acc[v] += p[v];
  }
  block_sum<NT, NACC>(acc, red);
  const double2 S = make_double2(red[0][0], red[0][1]);
  double2 s = make_double2(1., 0.);
  if (mode == 1) s = crecip(make_double2(S.x * a.dX * a.dP, S.y * a.dX * a.dP));
  else if (mode == 2) { const double d = a.dX * a.dP; s = crecip(make_double2(S.x * d, S.y * d)); }
  const double dXdP = a.dX * a.dP;
  double val = 0.;
  if (obs_row && threadIdx.x < NOBS)
    val = threadIdx.x == 0 ? (s.x * S.x - s.y * S.y) * dXdP : s.x * (dXdP * red[0][threadIdx.x + 1]);
  if (obs_row && a.partials_im) {
    // the reference takes the observables of the normalised complex W: Re(s Z) = s.x Re Z - s.y Im Z
    // for each moment sum Z (the s.y term matters where the step does not keep sum W real)
    __syncthreads();   // every thread has read red[0][] before block_sum rewrites it
    double im[NACC];
#pragma unroll
    for (int v = 0; v < NACC; ++v) im[v] = 0.;
    for (int i = threadIdx.x; i < a.n_partials; i += NT) {
      const double* q = a.partials_im + (size_t)i * NIM;
#pragma unroll
      for (int v = 0; v < NIM; ++v) im[v] += q[v];
    }
    block_sum<NT, NACC>(im, red);
    if (threadIdx.x >= 1 && threadIdx.x < NOBS) val -= s.y * (dXdP * red[0][threadIdx.x - 1]);
  }
  if (obs_row && threadIdx.x < NOBS) obs_row[threadIdx.x] = val;
  __syncthreads();   // red[] is reused by the caller
  return s;
}

__device__ __forceinline__ void accumulate_obs(double (&acc)[NACC], double2 v, double x, double p,
                                               double dV, double V0, double mass_exact) {
  const double w = v.x;
  acc[0] += v.x;
  acc[1] += v.y;
  acc[2] += w * x;
  acc[3] += w * (x * x);
  acc[4] += w * p;
  acc[5] += w * (p * p);
  acc[6] += w * (p * x);
  acc[7] += w * dV;
  acc[8] += w * (p * dV);
  acc[9] += w * (dV * x);
  acc[10] += w * ((p * p) / (2. * mass_exact) + V0);
  acc[11] += (w < 0.) ? w : 0.;
}

// Imaginary parts of the moment sums of accumulate_obs (slots 2..11 there, 0..9 here).
__device__ __forceinline__ void accumulate_obs_im(double (&im)[NACC], double2 v, double x, double p,
                                                  double dV, double V0, double mass_exact) {
  const double u = v.y;
  im[0] += u * x;
  im[1] += u * (x * x);
  im[2] += u * p;
  im[3] += u * (p * p);
  im[4] += u * (p * x);
  im[5] += u * dV;
  im[6] += u * (p * dV);
  im[7] += u * (dV * x);
  im[8] += u * ((p * p) / (2. * mass_exact) + V0);
  im[9] += (v.x < 0.) ? u : 0.;
}

// The CTA's imaginary moment sums into a.partials_im (after the real ones have been stored).
template <int NT>
__device__ __forceinline__ void store_partials_im(const WigArgs& a, double (&im)[NACC], double (*red)[NACC]) {
  __syncthreads();   // the real sums have been read out of red[0][]
  block_sum<NT, NACC>(im, red);
  if (threadIdx.x < NIM) a.partials_im[(size_t)blockIdx.x * NIM + threadIdx.x] = red[0][threadIdx.x];
}

// ------------------------------------------------------------------ kernels
// Partial sums over the whole grid (initial state, or any state): grid-stride.
template <int NX, int NP, int NT>
__device__ __forceinline__ void reduce_body(const WigArgs& a, const double2* __restrict__ W,
                                            double* __restrict__ partials) {
  __shared__ double red[NT / 32][NACC];
  double acc[NACC], im[NACC];
#pragma unroll
  for (int v = 0; v < NACC; ++v) acc[v] = im[v] = 0.;
  const bool with_im = a.partials_im != nullptr;
  for (int e = blockIdx.x * NT + threadIdx.x; e < NX * NP; e += gridDim.x * NT) {
    const int i = e / NX, j = e - i * NX;
    accumulate_obs(acc, W[e], a.x_tab[j], a.p_tab[i], a.dV_tab[j], a.V0_tab[j], a.mass_exact);
    if (with_im) accumulate_obs_im(im, W[e], a.x_tab[j], a.p_tab[i], a.dV_tab[j], a.V0_tab[j], a.mass_exact);
  }
  block_sum<NT, NACC>(acc, red);
  if (threadIdx.x < NACC) partials[(size_t)blockIdx.x * NACC + threadIdx.x] = red[0][threadIdx.x];
  if (with_im) store_partials_im<NT>(a, im, red);
}

// One CTA: the last sample's observables and the final scale.
template <int NT>
__device__ __forceinline__ void finalize_body(const WigArgs& a, int mode, double* obs_row,
                                              double2* scale_out) {
  __shared__ double red[NT / 32][NACC];
  const double2 s = consume_partials<NT>(a, mode, obs_row, red);
  if (threadIdx.x == 0) *scale_out = s;
}

template <int NT>
__device__ __forceinline__ void scale_body(double2* __restrict__ W, long n, const double2* s_ptr) {
  const double2 s = *s_ptr;
  for (long e = (long)blockIdx.x * NT + threadIdx.x; e < n; e += (long)gridDim.x * NT)
    W[e] = cmul(W[e], s);
}

// x-pass: ROWS rows per CTA.
template <class Phys, int NX, int NP, int ROWS, int NT, bool KIN_STRING>
__device__ __forceinline__ void xpass_body(const WigArgs& a, const Phys& ph, double2* __restrict__ W,
                                           int scale_mode, double* obs_row) {
  typedef RowMap<NX> M;
  extern __shared__ double2 sm[];
  __shared__ double red[NT / 32][NACC];
  double2 s = make_double2(1., 0.);
  if (scale_mode != 0 || (obs_row != nullptr && blockIdx.x == 0))
    s = consume_partials<NT>(a, scale_mode, blockIdx.x == 0 ? obs_row : nullptr, red);

  const int row0 = blockIdx.x * ROWS;
  WIG_BOUNDS_CHECK("x-pass rows", row0 + ROWS - 1, NP);
  double2* Wb = W + (size_t)row0 * NX;
  for (int e = threadIdx.x; e < ROWS * NX; e += NT) {
    const int r = e / NX, k = e - r * NX;
    double2 v = Wb[e];
    if (scale_mode != 0) v = cmul(v, s);
    sm[M::idx(r, k)] = v;
  }
  __syncthreads();
  cta_fft<double2, NX, ROWS, NT, false, M, WIG_XR>(sm, a.tw_x);
  const double inv_n = 1.0 / (double)NX;
  for (int e = threadIdx.x; e < ROWS * NX; e += NT) {
    const int r = e / NX, k = e - r * NX;
    const int ii = (row0 + r + NP / 2) % NP;
    const int jj = (k + NX / 2) % NX;
    const double lambda = a.dlambda * (jj - 0.5 * NX);
    const double p = a.dp * (ii - 0.5 * NP);
    double phase;
    if (KIN_STRING)
      phase = a.dt * ((ph.KineticEnergy(p + a.hbar * lambda / 2.) -
                       ph.KineticEnergy(p - a.hbar * lambda / 2.)) / a.hbar);
    else
      phase = a.dt * lambda * p / a.mass;
    const double rr = a.r_lambda[k] * inv_n;
    double sn, cs;
    sincos(phase, &sn, &cs);
    const int id = M::idx(r, k);
    sm[id] = cmul(sm[id], make_double2(rr * cs, -rr * sn));
  }
  __syncthreads();
  cta_fft<double2, NX, ROWS, NT, true, M, WIG_XR>(sm, a.tw_x);
  for (int e = threadIdx.x; e < ROWS * NX; e += NT) {
    const int r = e / NX, k = e - r * NX;
    Wb[e] = sm[M::idx(r, k)];
  }
}

// D(B) = IFFT_p[theta FFT_p(sign(p) f(p) B)] / n_p, in place on the tile;
// sfp / ths are the per-row factor tables staged in shared memory.
template <int NP, int C, int NT>
__device__ __forceinline__ void cl_apply_D(const WigArgs& a, double2* B, const double* sfp, const double* ths) {
  typedef ColMap<C> M;
  for (int e = threadIdx.x; e < C * NP; e += NT) B[pad8(e)] = cscale(B[pad8(e)], sfp[e / C]);
  __syncthreads();
  cta_fft<double2, NP, C, NT, false, M, WIG_PR>(B, a.tw_p);
  for (int e = threadIdx.x; e < C * NP; e += NT) B[pad8(e)] = cscale(B[pad8(e)], ths[e / C]);
  __syncthreads();
  cta_fft<double2, NP, C, NT, true, M, WIG_PR>(B, a.tw_p);
}

// p-pass: a tile of C columns x NP rows per CTA.  DAMP: 0 none, 1 Caldeira-Leggett.
// KVN: 0 the Moyal factor (expPotential_source :80-126), 1 the classical
// Liouville factor of GPU_FokkerPlank2D_FFT, phase dt (-V'(t, x) theta)
// (exp_PotentialKvN_source :27-75).
// Shared memory: A [padded C*NP], B [padded C*NP] and the two per-row CL
// tables [2*NP doubles] when DAMP == 1.
// Strang / Gross-Pitaevskii variant (GPU_Wigner2D_GPitaevskii.Run :1897-1975):
// HALF = 1 takes half the Moyal phase and exp(-0.5 D_Theta theta^2 dt)
// (expPotential_source Kernel :59-88); FINAL = 0 stops after the column IFFT
// (no damping, no partial sums).  scale_mode / obs_row: reduce the previous
// pass's partials, apply the pending normalisation on load and record that
// sample (the x-pass does this in the Lie step).  gp_phase (may be null): the
// Gross-Pitaevskii phase per (theta row, x column), applied as exp(i phase)
// (expPotential_GrossPitaevskii_source Kernel :466-495).
template <class Phys, int NX, int NP, int C, int NT, int DAMP, int KVN = 0, int HALF = 0, int FINAL = 1>
__device__ __forceinline__ void ppass_body(const WigArgs& a, const Phys& ph, double2* __restrict__ W,
                                           double t, double* __restrict__ partials, int scale_mode = 0,
                                           double* obs_row = nullptr, const double* __restrict__ gp_phase = nullptr) {
  typedef ColMap<C> M;
  constexpr int TILE = padded_size(C * NP);
  extern __shared__ double2 sm[];
  __shared__ double red[NT / 32][NACC];
  double2* A = sm;
  double2* B = sm + TILE;
  double* sfp = reinterpret_cast<double*>(sm + 2 * TILE);
  double* ths = sfp + NP;
  const int col0 = blockIdx.x * C;
  double2 s = make_double2(1., 0.);
  if (scale_mode != 0 || (obs_row != nullptr && blockIdx.x == 0))
    s = consume_partials<NT>(a, scale_mode, blockIdx.x == 0 ? obs_row : nullptr, red);
  if (DAMP == 1) {
    for (int k = threadIdx.x; k < NP; k += NT) { sfp[k] = a.sfp[k]; ths[k] = a.theta_s[k]; }
  }
  for (int e = threadIdx.x; e < C * NP; e += NT) {
    const int k = e / C, c = e - k * C;
    WIG_BOUNDS_CHECK("p-pass tile column", col0 + c, NX);
    double2 v = W[(size_t)k * NX + col0 + c];
    if (scale_mode != 0) v = cmul(v, s);
    A[pad8(e)] = v;
  }
  __syncthreads();
  cta_fft<double2, NP, C, NT, false, M, WIG_PR>(A, a.tw_p);
  for (int e = threadIdx.x; e < C * NP; e += NT) {
    const int k = e / C, c = e - k * C;
    const int col = col0 + c;
    const int ii = (k + NP / 2) % NP;
    const int jj = (col + NX / 2) % NX;
    const double x = a.dx * (jj - 0.5 * NX);
    const double theta = a.dtheta * (ii - 0.5 * NP);
    const double phase = KVN ? a.dt * (-ph.DPotential(t, x) * theta)
                       : (HALF ? 0.5 * a.dt : a.dt) * ((ph.Potential(t, x - a.hbar * theta / 2.) -
                                                        ph.Potential(t, x + a.hbar * theta / 2.)) / a.hbar);
    const double r = HALF ? a.r_theta_half[k] : a.r_theta[k];
    double sn, cs;
    sincos(phase, &sn, &cs);
    double2 v = cmul(A[pad8(e)], make_double2(r * cs, -r * sn));
    v = cscale(v, a.mask1[col]);
    v = cscale(v, a.mask2s[col]);
    if (gp_phase != nullptr) {
      double gs, gc;
      sincos(gp_phase[(size_t)k * NX + col], &gs, &gc);
      v = cmul(v, make_double2(gc, gs));
    }
    A[pad8(e)] = v;
  }
  __syncthreads();
  cta_fft<double2, NP, C, NT, true, M, WIG_PR>(A, a.tw_p);
  if (!FINAL) {
    for (int e = threadIdx.x; e < C * NP; e += NT) {
      const int k = e / C, c = e - k * C;
      W[(size_t)k * NX + col0 + c] = A[pad8(e)];
    }
    return;
  }
  if (DAMP == 1) {
    for (int e = threadIdx.x; e < C * NP; e += NT) B[pad8(e)] = A[pad8(e)];
    cl_apply_D<NP, C, NT>(a, B, sfp, ths);
    for (int e = threadIdx.x; e < C * NP; e += NT) B[pad8(e)] = cadd(A[pad8(e)], cmul(a.cl_k1, B[pad8(e)]));
    cl_apply_D<NP, C, NT>(a, B, sfp, ths);
    for (int e = threadIdx.x; e < C * NP; e += NT) B[pad8(e)] = cadd(A[pad8(e)], cmul(a.cl_k12, B[pad8(e)]));
    cl_apply_D<NP, C, NT>(a, B, sfp, ths);
    for (int e = threadIdx.x; e < C * NP; e += NT) A[pad8(e)] = cadd(A[pad8(e)], cmul(a.cl_c3, B[pad8(e)]));
    __syncthreads();
  }
  double acc[NACC];
#pragma unroll
  for (int v = 0; v < NACC; ++v) acc[v] = 0.;
  for (int e = threadIdx.x; e < C * NP; e += NT) {
    const int k = e / C, c = e - k * C;
    const int col = col0 + c;
    const double2 v = A[pad8(e)];
    W[(size_t)k * NX + col] = v;
    accumulate_obs(acc, v, a.x_tab[col], a.p_tab[k], a.dV_tab[col], a.V0_tab[col], a.mass_exact);
  }
  block_sum<NT, NACC>(acc, red);
  if (threadIdx.x < NACC) partials[(size_t)blockIdx.x * NACC + threadIdx.x] = red[0][threadIdx.x];
}

// ------------------------------------------------------------------ Gross-Pitaevskii terms
// (MakeGrossPitaevskiiTerms :1717-1736 with ProbabilityX :1743-1748)
// Column sums of W over a chunk of RCH rows: out[chunk][x] (grid NX/NT x NP/RCH).
template <int NX, int NP, int RCH, int NT>
__device__ __forceinline__ void colsum_body(const double2* __restrict__ W, double2* __restrict__ out) {
  const int x = blockIdx.x * NT + threadIdx.x, r0 = blockIdx.y * RCH;
  if (x >= NX) return;
  double sr = 0., si = 0.;
#pragma unroll 8
  for (int r = 0; r < RCH; ++r) {
    const double2 v = W[(size_t)(r0 + r) * NX + x];
    sr += v.x;
    si += v.y;
  }
  out[(size_t)blockIdx.y * NX + x] = make_double2(sr, si);
}

// P(x) = dP Re(s sum_p W) from the chunk sums (fixed order), s the pending
// normalisation of scale_mode (1 / 2 as consume_partials, 0: none); one CTA.
// psq (may be null) = sum_x P(x)^2 dX (ProbabilitySquare_average, :1951).
template <int NX, int NT>
__device__ __forceinline__ void gp_marginal_body(const WigArgs& a, const double2* __restrict__ chunks,
                                                 int n_chunks, int scale_mode, double* __restrict__ P,
                                                 double* __restrict__ psq) {
  __shared__ double red[NT / 32][NACC];
  const double2 s = consume_partials<NT>(a, scale_mode, nullptr, red);
  double acc[NACC];
#pragma unroll
  for (int v = 0; v < NACC; ++v) acc[v] = 0.;
  for (int x = threadIdx.x; x < NX; x += NT) {
    double sr = 0., si = 0.;
    for (int c = 0; c < n_chunks; ++c) {
      const double2 v = chunks[(size_t)c * NX + x];
      sr += v.x;
      si += v.y;
    }
    const double px = a.dP * (s.x * sr - s.y * si);
    P[x] = px;
    acc[0] += px * px;
  }
  block_sum<NT, NACC>(acc, red);
  if (psq != nullptr && threadIdx.x == 0) *psq = red[0][0] * a.dX;
}

// Gross-Pitaevskii phase of ROWS theta rows per CTA:
//   phase(theta_i, x) = -0.5 dt a_GP Re[P(x - theta_i/2) - P(x + theta_i/2)] / hbar,
// the shifted marginals by the shift theorem on the exact Lambda / Theta grids:
// Re IFFT_x[FFT_x(P) (-2 i sin(lambda theta_i / 2))] / N_x.
template <int NX, int NP, int ROWS, int NT>
__device__ __forceinline__ void gp_phase_body(const WigArgs& a, const double* __restrict__ P,
                                              double* __restrict__ phase_out) {
  typedef RowMap<NX> M;
  extern __shared__ double2 sm[];
  double2* Ph = sm;                              // FFT of the marginal (one sequence)
  double2* R = sm + padded_size(NX);             // ROWS rows
  for (int x = threadIdx.x; x < NX; x += NT) Ph[M::idx(0, x)] = make_double2(P[x], 0.);
  __syncthreads();
  cta_fft<double2, NX, 1, NT, false, M>(Ph, a.tw_x);
  const int row0 = blockIdx.x * ROWS;
  for (int e = threadIdx.x; e < ROWS * NX; e += NT) {
    const int r = e / NX, k = e - r * NX;
    const double th = a.theta_s[row0 + r] * (double)NP;    // exact shifted Theta
    const double sn = sin(0.5 * a.lambda_tab[k] * th);
    const double2 f = Ph[M::idx(0, k)];
    R[M::idx(r, k)] = make_double2(2. * sn * f.y, -2. * sn * f.x);
  }
  __syncthreads();
  cta_fft<double2, NX, ROWS, NT, true, M>(R, a.tw_x);
  const double c = -0.5 * a.dt * a.gp_coef / a.hbar * (1.0 / (double)NX);
  for (int e = threadIdx.x; e < ROWS * NX; e += NT) {
    const int r = e / NX, k = e - r * NX;
    phase_out[(size_t)(row0 + r) * NX + k] = c * R[M::idx(r, k)].x;
  }
}

// ------------------------------------------------------------------ Bloch (imaginary time)
// GPU_Wigner2D_GPitaevskii_Bloch (:2064-2342): the Strang step with real
// exponentials and a run-time step dtb (Kernel_Bloch of expPotential_source
// :90-114 and expPLambdaKinetic_source :155-178).
// p-half: W(theta, x) *= exp(-0.25 dtb [V(x - hbar theta/2) + V(x + hbar theta/2)])
//         * exp(gexp(theta, x)) (mean-field, may be null); no masks, no diffusion.
template <class Phys, int NX, int NP, int C, int NT>
__device__ __forceinline__ void bloch_ppass_body(const WigArgs& a, const Phys& ph, double2* __restrict__ W,
                                                 double t, double dtb, const double* __restrict__ gexp) {
  typedef ColMap<C> M;
  extern __shared__ double2 sm[];
  double2* A = sm;
  const int col0 = blockIdx.x * C;
  for (int e = threadIdx.x; e < C * NP; e += NT) {
    const int k = e / C, c = e - k * C;
    WIG_BOUNDS_CHECK("ODM p-pass tile column", col0 + c, NX);
    A[pad8(e)] = W[(size_t)k * NX + col0 + c];
  }
  __syncthreads();
  cta_fft<double2, NP, C, NT, false, M>(A, a.tw_p);
  const double inv_n = 1.0 / (double)NP;
  for (int e = threadIdx.x; e < C * NP; e += NT) {
    const int k = e / C, c = e - k * C;
    const int col = col0 + c;
    const int ii = (k + NP / 2) % NP, jj = (col + NX / 2) % NX;
    const double x = a.dx * (jj - 0.5 * NX);
    const double theta = a.dtheta * (ii - 0.5 * NP);
    double f = exp(-0.25 * dtb * (ph.Potential(t, x - a.hbar * theta / 2.) + ph.Potential(t, x + a.hbar * theta / 2.)));
    if (gexp != nullptr) f *= exp(gexp[(size_t)k * NX + col]);
    A[pad8(e)] = cscale(A[pad8(e)], f * inv_n);
  }
  __syncthreads();
  cta_fft<double2, NP, C, NT, true, M>(A, a.tw_p);
  for (int e = threadIdx.x; e < C * NP; e += NT) {
    const int k = e / C, c = e - k * C;
    W[(size_t)k * NX + col0 + c] = A[pad8(e)];
  }
}

// x-pass: W(p, lambda) *= exp(-0.5 dtb [K(p + hbar lambda/2) + K(p - hbar lambda/2)]).
template <class Phys, int NX, int NP, int ROWS, int NT>
__device__ __forceinline__ void bloch_xpass_body(const WigArgs& a, const Phys& ph, double2* __restrict__ W,
                                                 double dtb) {
  typedef RowMap<NX> M;
  extern __shared__ double2 sm[];
  const int row0 = blockIdx.x * ROWS;
  WIG_BOUNDS_CHECK("x-pass rows", row0 + ROWS - 1, NP);
  double2* Wb = W + (size_t)row0 * NX;
  for (int e = threadIdx.x; e < ROWS * NX; e += NT) {
    const int r = e / NX, k = e - r * NX;
    sm[M::idx(r, k)] = Wb[e];
  }
  __syncthreads();
  cta_fft<double2, NX, ROWS, NT, false, M>(sm, a.tw_x);
  const double inv_n = 1.0 / (double)NX;
  for (int e = threadIdx.x; e < ROWS * NX; e += NT) {
    const int r = e / NX, k = e - r * NX;
    const int ii = (row0 + r + NP / 2) % NP, jj = (k + NX / 2) % NX;
    const double lambda = a.dlambda * (jj - 0.5 * NX);
    const double p = a.dp * (ii - 0.5 * NP);
    const double f = exp(-0.5 * dtb * (ph.KineticEnergy(p + a.hbar * lambda / 2.) +
                                      ph.KineticEnergy(p - a.hbar * lambda / 2.)));
    const int id = M::idx(r, k);
    sm[id] = cscale(sm[id], f * inv_n);
  }
  __syncthreads();
  cta_fft<double2, NX, ROWS, NT, true, M>(sm, a.tw_x);
  for (int e = threadIdx.x; e < ROWS * NX; e += NT) {
    const int r = e / NX, k = e - r * NX;
    Wb[e] = sm[M::idx(r, k)];
  }
}

// Mean-field exponent of Kernel_Bloch (expPotential_GrossPitaevskii_source
// :497-517): -0.25 dtb a_GP [P(x - theta/2) + P(x + theta/2)], the shifted
// marginals summed by the shift theorem: Re IFFT_x[FFT_x(P) 2 cos(lambda theta/2)] / N_x.
template <int NX, int NP, int ROWS, int NT>
__device__ __forceinline__ void gp_bloch_body(const WigArgs& a, const double* __restrict__ P, double dtb,
                                              double* __restrict__ out) {
  typedef RowMap<NX> M;
  extern __shared__ double2 sm[];
  double2* Ph = sm;
  double2* R = sm + padded_size(NX);
  for (int x = threadIdx.x; x < NX; x += NT) Ph[M::idx(0, x)] = make_double2(P[x], 0.);
  __syncthreads();
  cta_fft<double2, NX, 1, NT, false, M>(Ph, a.tw_x);
  const int row0 = blockIdx.x * ROWS;
  for (int e = threadIdx.x; e < ROWS * NX; e += NT) {
    const int r = e / NX, k = e - r * NX;
    const double th = a.theta_s[row0 + r] * (double)NP;
    const double cs = 2. * cos(0.5 * a.lambda_tab[k] * th);
    const double2 f = Ph[M::idx(0, k)];
    R[M::idx(r, k)] = make_double2(cs * f.x, cs * f.y);
  }
  __syncthreads();
  cta_fft<double2, NX, ROWS, NT, true, M>(R, a.tw_x);
  const double c = -0.25 * dtb * a.gp_coef * (1.0 / (double)NX);
  for (int e = threadIdx.x; e < ROWS * NX; e += NT) {
    const int r = e / NX, k = e - r * NX;
    out[(size_t)(row0 + r) * NX + k] = c * R[M::idx(r, k)].x;
  }
}

// Observables of a Bloch step (one CTA per block of the grid, partials per CTA):
// sums of W, W x, W x^2, W p, W p^2, W [K(p) + V(0, x)] (the Bloch Hamiltonian,
// :2097 -- the kinetic string, not p^2/2m), W^2 (purity, Purity_GPU :1738-1741),
// W W0 (ExitedState1 projection, :2431) and the p-marginal rows are separate.
constexpr int NBL = 12;   // Re/Im sum, x, x2, p, p2, H, Re/Im W^2, Re/Im W W0, spare
template <class Phys, int NX, int NP, int NT>
__device__ __forceinline__ void bloch_reduce_body(const WigArgs& a, const Phys& ph, const double2* __restrict__ W,
                                                  const double2* __restrict__ W0, double* __restrict__ partials) {
  __shared__ double red[NT / 32][NBL];
  double acc[NBL];
#pragma unroll
  for (int v = 0; v < NBL; ++v) acc[v] = 0.;
  for (int e = blockIdx.x * NT + threadIdx.x; e < NX * NP; e += gridDim.x * NT) {
    const int i = e / NX, j = e - i * NX;
    const double2 v = W[e];
    const double x = a.x_tab[j], p = a.p_tab[i];
    acc[0] += v.x; acc[1] += v.y;
    acc[2] += v.x * x; acc[3] += v.x * (x * x);
    acc[4] += v.x * p; acc[5] += v.x * (p * p);
    acc[6] += v.x * (ph.KineticEnergy(p) + a.V0_tab[j]);
    acc[7] += v.x * v.x - v.y * v.y; acc[8] += 2. * v.x * v.y;
    if (W0 != nullptr) {
      const double2 u = W0[e];
      acc[9] += v.x * u.x - v.y * u.y; acc[10] += v.x * u.y + v.y * u.x;
    }
  }
  block_sum<NT, NBL>(acc, red);
  if (threadIdx.x < NBL) partials[(size_t)blockIdx.x * NBL + threadIdx.x] = red[0][threadIdx.x];
}

// Row sums of W (the p-marginal): out[i] = sum_x W[i][x] (ProbabilityP :1750-1755).
template <int NX, int NT>
__device__ __forceinline__ void rowsum_body(const double2* __restrict__ W, double2* __restrict__ out) {
  __shared__ double red[NT / 32][2];
  double acc[2] = {0., 0.};
  const double2* r = W + (size_t)blockIdx.x * NX;
  for (int j = threadIdx.x; j < NX; j += NT) { acc[0] += r[j].x; acc[1] += r[j].y; }
  block_sum<NT, 2>(acc, red);
  if (threadIdx.x == 0) out[blockIdx.x] = make_double2(red[0][0], red[0][1]);
}

// W <- s (W - c W0)  (projection and normalisation of a Bloch step)
template <int NT>
__device__ __forceinline__ void bloch_axpy_body(double2* __restrict__ W, const double2* __restrict__ W0,
                                                long n, double2 c, double2 s) {
  for (long e = (long)blockIdx.x * NT + threadIdx.x; e < n; e += (long)gridDim.x * NT) {
    double2 v = W[e];
    if (W0 != nullptr) v = csub(v, cmul(c, W0[e]));
    W[e] = cmul(v, s);
  }
}

// ------------------------------------------------------------------ ODM Lindblad
// g_ODM(p) = sqrt(L f(|p| + hbar/(2L)))  (g_ODM :1196-1197); the five
// momentum-space factor combinations of _Lindbladian_ODM (:1524-1623), with
// the two gg terms (:1602-1623) summed: T_k = IFFT_x[FFT_x(W) G_k] / n_x.
template <class Phys>
__device__ __forceinline__ double odm_g(const WigArgs& a, const Phys& ph, double p) {
  return sqrt(a.L_material * ph.f(fabs(p) + a.hbar_exact / (2. * a.L_material)));
}

__device__ __forceinline__ double sgn(double v) { return v > 0. ? 1. : (v < 0. ? -1. : 0.); }

template <class Phys, int NX, int NP, int ROWS, int NT>
__device__ __forceinline__ void odm_xpass_body(const WigArgs& a, const Phys& ph, const double2* __restrict__ W,
                                               double2* __restrict__ T) {
  typedef RowMap<NX> M;
  extern __shared__ double2 sm[];
  double2* F = sm;                                 // FFT_x(W) of the CTA's rows
  double2* B = sm + padded_size(ROWS * NX);        // one factor combination at a time
  const int row0 = blockIdx.x * ROWS;
  const double2* Wb = W + (size_t)row0 * NX;
  for (int e = threadIdx.x; e < ROWS * NX; e += NT) {
    const int r = e / NX, k = e - r * NX;
    F[M::idx(r, k)] = Wb[e];
  }
  __syncthreads();
  cta_fft<double2, NX, ROWS, NT, false, M>(F, a.tw_x);
  const double inv_n = 1.0 / (double)NX;
  const size_t plane = (size_t)NX * NP;
#pragma unroll 1
  for (int term = 0; term < 5; ++term) {
    for (int e = threadIdx.x; e < ROWS * NX; e += NT) {
      const int r = e / NX, k = e - r * NX;
      const double p = a.p_tab[row0 + r], lam = a.lambda_tab[k];
      const double pp = p + 0.5 * a.hbar_exact * lam, pm = p - 0.5 * a.hbar_exact * lam;
      const double gp = odm_g(a, ph, pp), gm = odm_g(a, ph, pm);
      double m;
      if (term == 0) m = gp * gm;
      else if (term == 1) m = gp * (gm * sgn(pm));
      else if (term == 2) m = (gp * sgn(pp)) * gm;
      else if (term == 3) m = (gp * sgn(pp)) * (gm * sgn(pm));
      else m = -0.5 * gp * gp + -0.5 * gm * gm;
      const int id = M::idx(r, k);
      B[id] = cscale(F[id], m * inv_n);
    }
    __syncthreads();
    cta_fft<double2, NX, ROWS, NT, true, M>(B, a.tw_x);
    double2* Tk = T + term * plane + (size_t)row0 * NX;
    for (int e = threadIdx.x; e < ROWS * NX; e += NT) {
      const int r = e / NX, k = e - r * NX;
      Tk[e] = B[M::idx(r, k)];
    }
    __syncthreads();
  }
}

// ODM p-pass: W <- W + coef * IFFT_p[ sum_k trig_k(x, theta) FFT_p(T_k) ]
// (trig factors of SetA_ODM from the exact X, Theta tables; coef =
// dt 2 gamma weight / n / n_p folded), then the observable partial sums.
template <int NX, int NP, int C, int NT>
__device__ __forceinline__ void odm_ppass_body(const WigArgs& a, double2* __restrict__ W,
                                               const double2* __restrict__ T, double coef, double sign) {
  typedef ColMap<C> M;
  extern __shared__ double2 sm[];
  __shared__ double red[NT / 32][NACC];
  double2* Acc = sm;
  double2* B = sm + padded_size(C * NP);
  const int col0 = blockIdx.x * C;
  const size_t plane = (size_t)NX * NP;
  for (int e = threadIdx.x; e < C * NP; e += NT) Acc[pad8(e)] = make_double2(0., 0.);
#pragma unroll 1
  for (int term = 0; term < 5; ++term) {
    const double2* Tk = T + term * plane;
    for (int e = threadIdx.x; e < C * NP; e += NT) {
      const int k = e / C, c = e - k * C;
      B[pad8(e)] = Tk[(size_t)k * NX + col0 + c];
    }
    __syncthreads();
    cta_fft<double2, NP, C, NT, false, M>(B, a.tw_p);
    for (int e = threadIdx.x; e < C * NP; e += NT) {
      const int k = e / C, c = e - k * C;
      const double X = a.x_tab[col0 + c], Th = a.theta_s[k] * (double)NP;
      const double xp = X + 0.5 * a.hbar_exact * Th, xm = X - 0.5 * a.hbar_exact * Th;
      double2 v = B[pad8(e)];
      if (term == 0) {
        v = cscale(v, cos(xp) * cos(xm));
      } else if (term == 1) {
        v = cscale(cscale(v, cos(xm)), sin(xp));
        v = cmul(v, make_double2(0., sign));
      } else if (term == 2) {
        v = cscale(cscale(v, sin(xm)), cos(xp));
        v = cmul(v, make_double2(0., -sign));
      } else if (term == 3) {
        v = cscale(v, sin(xp) * sin(xm));
      }
      Acc[pad8(e)] = cadd(Acc[pad8(e)], v);
    }
    __syncthreads();
  }
  cta_fft<double2, NP, C, NT, true, M>(Acc, a.tw_p);
  double acc[NACC], im[NACC];
#pragma unroll
  for (int v = 0; v < NACC; ++v) acc[v] = im[v] = 0.;
  const bool with_im = a.partials_im != nullptr;
  for (int e = threadIdx.x; e < C * NP; e += NT) {
    const int k = e / C, c = e - k * C;
    const int col = col0 + c;
    const size_t g = (size_t)k * NX + col;
    const double2 v = cadd(W[g], cscale(Acc[pad8(e)], coef));
    W[g] = v;
    accumulate_obs(acc, v, a.x_tab[col], a.p_tab[k], a.dV_tab[col], a.V0_tab[col], a.mass_exact);
    if (with_im) accumulate_obs_im(im, v, a.x_tab[col], a.p_tab[k], a.dV_tab[col], a.V0_tab[col], a.mass_exact);
  }
  block_sum<NT, NACC>(acc, red);
  if (threadIdx.x < NACC) a.partials[(size_t)blockIdx.x * NACC + threadIdx.x] = red[0][threadIdx.x];
  if (with_im) store_partials_im<NT>(a, im, red);
}

}  // namespace wig

