// Adjoint (differentiable) FP32 Wigner2D form: one grid, the Lie step
// W_{n+1} = P(eps_n) K W_n of GPU_Wigner2D_FFT.Run (:1884-1899) with
//   K       x-pass: IFFT_x[ r_lambda(lambda) e^{-i dt lambda p / m} FFT_x W ] / N_x
//   P(eps)  p-pass: IFFT_p[ r_theta(theta) mask(x) e^{-i dt [V(x - u) - V(x + u)] / hbar} FFT_p Y ] / N_p,
//           u = hbar theta / 2,  V(x) = v4 x^4 + v2 x^2 + v0 + eps_n x  (eps_n: a control per step)
// and its adjoint.  Both passes are complex-linear, so for the real inner
// product <A, B> = Re sum conj(A) B the adjoint of F^H diag(d) F (F the
// unnormalised DFT) is F^H diag(conj d) F: the adjoint step is the same pair of
// passes in reverse order with conjugated factors.  With Y_n = K W_n kept from
// the forward sweep, the adjoint p-pass also gives
//   dL/d eps_n = Re <lambda_{n+1}, dP/d eps Y_n> = Re sum_k conj(F lambda)_k (i dt theta_k) d_k (F Y)_k
// per column (dP/d eps multiplies the theta-space factor d_k by i dt theta_k).
// No counterpart in the reference (it has no gradients).
#pragma once
#include "wig_rfft.cuh"
#include "wig_wigner.cuh"

namespace wig {

struct AArgs {
  int n_x, n_p;
  double dt, hbar, mass, dx, dp, dtheta, dlambda;
  double v4, v2, v0;
  const float2* tw_x;   // register-FFT twiddles of n_x (2 n_x entries: forward, inverse)
  const float2* tw_p;   // of n_p
  const float* rtab;    // [n_x] exp(-D_lambda lambda^2) / n_x       (per frequency)
  const float* mm;      // [n_x] mask1 mask2 / n_p                    (per column)
  const float* rth;     // [n_p] exp(-D_theta theta^2 dt)            (per frequency)
};

__device__ __forceinline__ int ashift(int k, int n) { return k < n / 2 ? k : k - n; }

// e^{-2 pi i s t} r, t reduced to one turn in FP64 (s = +-1)
__device__ __forceinline__ float2 adj_turn(double t, float r, float s) {
  const float f = (float)(t - rint(t));
  float sn, cs;
  sincospif(2.f * f, &sn, &cs);
  return make_float2(r * cs, -s * r * sn);
}

// Column c of a CT-wide tile owned by group `grp` of warp `warp` (tile of
// WARPS * rf_spw(N) columns); 8-lane groups pair columns c and c ^ PM so the
// two sequences of a half-warp use distinct bank pairs.
template <int N, int WARPS>
__device__ __forceinline__ int adj_col(int warp, int grp) {
  constexpr int G = rf_g(N), SPW = rf_spw(N), CT = WARPS * SPW;
  if constexpr (G == 8) {
    constexpr int PM = CT / 2 < 8 ? CT / 2 : 8;
    const int hw = 2 * warp + (grp >> 1);
    const int base = (hw & (PM - 1)) | ((hw / PM) * 2 * PM);
    return base ^ ((grp & 1) * PM);
  } else {
    return warp * SPW + grp;
  }
}

// x-pass, one warp per CTA, rf_spw(NX) rows per warp: out = K in (sgn = +1)
// or K^H in (sgn = -1); in and out may alias.
template <int NX, int NP>
__device__ __forceinline__ void adj_xpass(const AArgs& a, const float2* in, float2* out, float sgn) {
  typedef RegFft<float2, NX> F;
  constexpr int E = F::E, G = F::G, Q = F::Q, SPW = rf_spw(NX);
  constexpr int XS = NX + (G == 8 ? 8 : 0);
  extern __shared__ float2 sma[];
  const int lane = threadIdx.x & 31, grp = lane / G, g = lane % G;
  const int row = blockIdx.x * SPW + grp;
  const float2* src = in + (size_t)row * NX;
  float2 v[E];
#pragma unroll
  for (int m = 0; m < E; ++m) v[m] = src[g + G * m];
  const PlainSlot sl{grp * XS};
  F::fwd(v, sma, sl, a.tw_x, g);
  const double cq = a.dt * a.dp * a.dlambda * (double)ashift(row, NP) / (a.mass * 6.283185307179586477);
#pragma unroll
  for (int i = 0; i < Q; ++i)
#pragma unroll
    for (int b = 0; b < G; ++b) {
      const int k = g * Q + i + E * b;
      const int lj = b < G / 2 ? k : k - NX;
      v[i * G + b] = cmul(v[i * G + b], adj_turn(cq * (double)lj, __ldg(a.rtab + k), sgn));
    }
  F::inv(v, sma, sl, a.tw_x + NX, g);
  float2* dst = out + (size_t)row * NX;
#pragma unroll
  for (int m = 0; m < E; ++m) dst[g + G * m] = v[m];
}

// theta-space turn count of the Moyal factor at signed index j for column x:
// t = j (al + be j^2), the phase exp(-2 pi i t); returns al, be for x and eps.
__device__ __forceinline__ void moyal_coeffs(const AArgs& a, double x, double eps, double* al, double* be) {
  const double h = 0.5 * a.hbar * a.dtheta;
  const double kk = -a.dt * h / (3.141592653589793238 * a.hbar);
  *al = kk * ((4. * a.v4 * x * x + 2. * a.v2) * x + eps);
  *be = kk * h * h * (4. * a.v4 * x);
}

// Coalesced load of a CT x NP tile of columns [col0, col0 + CT) into the swizzled tile.
template <int NP, int CT, int NT>
__device__ __forceinline__ void adj_tile_load(float2* tile, const float2* src, int nx, int col0) {
  for (int e = threadIdx.x; e < CT * NP; e += NT) {
    const int k = e / CT, c = e & (CT - 1);
    tile[k * CT + (c ^ tile_sw<CT>(k))] = src[(size_t)k * nx + col0 + c];
  }
}
template <int NP, int CT, int NT>
__device__ __forceinline__ void adj_tile_store(const float2* tile, float2* dst, int nx, int col0) {
  for (int e = threadIdx.x; e < CT * NP; e += NT) {
    const int k = e / CT, c = e & (CT - 1);
    dst[(size_t)k * nx + col0 + c] = tile[k * CT + (c ^ tile_sw<CT>(k))];
  }
}

// Forward p-pass (in place allowed): out = P(eps_step) in.
template <int NX, int NP, int WARPS>
__device__ __forceinline__ void adj_ppass(const AArgs& a, const float2* in, float2* out, double eps) {
  typedef RegFft<float2, NP> F;
  constexpr int E = F::E, G = F::G, Q = F::Q, SPW = rf_spw(NP), CT = WARPS * SPW, NT = WARPS * 32;
  extern __shared__ float2 sma[];
  float2* tile = sma;
  const int col0 = blockIdx.x * CT;
  adj_tile_load<NP, CT, NT>(tile, in, NX, col0);
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, grp = lane / G, g = lane % G;
  const int c = adj_col<NP, WARPS>(warp, grp);
  const TileSlot<CT> sl{c};
  float2 w[E];
#pragma unroll
  for (int m = 0; m < E; ++m) w[m] = tile[sl(g + G * m)];
  F::fwd(w, tile, sl, a.tw_p, g);
  const int col = col0 + c;
  double al, be;
  moyal_coeffs(a, a.dx * (double)ashift(col, NX), eps, &al, &be);
  const float mm = __ldg(a.mm + col);
#pragma unroll
  for (int i = 0; i < Q; ++i)
#pragma unroll
    for (int b = 0; b < G; ++b) {
      const int k = g * Q + i + E * b;
      const double j = (double)(b < G / 2 ? k : k - NP);
      w[i * G + b] = cmul(w[i * G + b], adj_turn(j * fma(be, j * j, al), __ldg(a.rth + k) * mm, 1.f));
    }
  F::inv(w, tile, sl, a.tw_p + NP, g);
  __syncwarp();
#pragma unroll
  for (int m = 0; m < E; ++m) tile[sl(g + G * m)] = w[m];
  __syncthreads();
  adj_tile_store<NP, CT, NT>(tile, out, NX, col0);
}

// Adjoint p-pass: lam <- P(eps)^H lam, and this CTA's share of
// dL/d eps = Re sum conj(F lam) (i dt theta) d (F Y) into partials[blockIdx.x].
template <int NX, int NP, int WARPS>
__device__ __forceinline__ void adj_ppass_T(const AArgs& a, float2* lam, const float2* Y, double eps,
                                            double* partials) {
  typedef RegFft<float2, NP> F;
  constexpr int E = F::E, G = F::G, Q = F::Q, SPW = rf_spw(NP), CT = WARPS * SPW, NT = WARPS * 32;
  extern __shared__ float2 sma[];
  float2* tl = sma;            // lambda tile
  float2* ty = sma + CT * NP;  // Y tile
  const int col0 = blockIdx.x * CT;
  adj_tile_load<NP, CT, NT>(tl, lam, NX, col0);
  adj_tile_load<NP, CT, NT>(ty, Y, NX, col0);
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, grp = lane / G, g = lane % G;
  const int c = adj_col<NP, WARPS>(warp, grp);
  const TileSlot<CT> sl{c};
  float2 u[E], y[E];
#pragma unroll
  for (int m = 0; m < E; ++m) { u[m] = tl[sl(g + G * m)]; y[m] = ty[sl(g + G * m)]; }
  F::fwd(u, tl, sl, a.tw_p, g);
  F::fwd(y, ty, sl, a.tw_p, g);
  const int col = col0 + c;
  double al, be;
  moyal_coeffs(a, a.dx * (double)ashift(col, NX), eps, &al, &be);
  const float mm = __ldg(a.mm + col);
  const double gth = a.dt * a.dtheta;   // d(phase)/d eps = dt theta = dt dtheta j
  double gacc = 0.;
#pragma unroll
  for (int i = 0; i < Q; ++i)
#pragma unroll
    for (int b = 0; b < G; ++b) {
      const int k = g * Q + i + E * b;
      const int ji = b < G / 2 ? k : k - NP;
      const double j = (double)ji;
      const float2 d = adj_turn(j * fma(be, j * j, al), __ldg(a.rth + k) * mm, 1.f);
      const float2 yd = cmul(y[i * G + b], d);
      const float2 U = u[i * G + b];
      // Re(conj(U) * i * yd) = U.x * (-yd.y) ... = U.y * yd.x - U.x * yd.y
      gacc += (double)ji * ((double)U.y * (double)yd.x - (double)U.x * (double)yd.y);
      u[i * G + b] = cmul(U, make_float2(d.x, -d.y));
    }
  gacc *= gth;
  F::inv(u, tl, sl, a.tw_p + NP, g);
  __syncwarp();
#pragma unroll
  for (int m = 0; m < E; ++m) tl[sl(g + G * m)] = u[m];
  // CTA sum of gacc in a fixed order
  __shared__ double red[32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) gacc += __shfl_xor_sync(0xffffffffu, gacc, o);
  if (lane == 0) red[warp] = gacc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.;
    for (int w = 0; w < WARPS; ++w) s += red[w];
    partials[blockIdx.x] = s;
  }
  adj_tile_store<NP, CT, NT>(tl, lam, NX, col0);
}

}  // namespace wig
