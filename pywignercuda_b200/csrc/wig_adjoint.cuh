// Adjoint (differentiable) Wigner2D form: one grid, the Lie step of
// GPU_Wigner2D_FFT.Run (:1884-1913)
//   Y_n     = K W_n                                     x-pass
//   A_n     = P(eps_n) Y_n                              p-pass, Moyal part
//   U_n     = C A_n            (damped only)            p-pass, Caldeira-Leggett order 3
//   W_{n+1} = U_n / s_n,  s_n = dX dP sum U_n   (damped only; undamped: W_{n+1} = A_n)
// with
//   K       IFFT_x[ r_lambda(lambda) e^{-i dt lambda p / m} FFT_x . ] / N_x
//   P(eps)  IFFT_p[ r_theta(theta) mask(x) e^{-i dt [V(x - u) - V(x + u)] / hbar} FFT_p . ] / N_p,
//           u = hbar theta / 2,  V(x) = v4 x^4 + v2 x^2 + v0 + eps_n x  (eps_n: a control per step)
//   C       I + a3 D (I + a2 D (I + a1 D)),  D = IFFT_p[ theta FFT_p(sign(p) f(p) .) ] / N_p,
//           a1 = i c1 c2 / (c1 + c2), a2 = i (c1 + c2), a3 = i c3, (c1, c2, c3) = (2/3, 1, 2) gamma dt
//           (CaldeiraDissipatorOrder3 :1145-1157 in Horner form),
// and its adjoint.  K, P and C are complex-linear, so for the real inner
// product <A, B> = Re sum conj(A) B the adjoint of F^H diag(d) F (F the
// unnormalised DFT) is F^H diag(conj d) F, and
//   C^H = I + conj(a3) D^H (I + conj(a2) D^H (I + conj(a1) D^H)),  D^H = sign(p) f(p) IFFT_p[ theta FFT_p . ] / N_p.
// The normalisation N(U) = U / (dX dP sum U) has the adjoint
//   lam_U = lam / conj(s) - conj(beta),  beta = dX dP (sum conj(lam) U) / s^2
// (a uniform shift: wiga_dot forms the sum, wiga_adj_coef the two scalars).
// With Y_n kept from the forward sweep, the adjoint p-pass also gives
//   dL/dq = Re <lam_A, dP/dq Y_n> = sum_k w_q(k, x) Re(i conj(F lam_A)_k d_k (F Y)_k)
// per column, for q = eps_n (w = dt theta), v4 (w = 8 dt x u (x^2 + u^2) / hbar)
// and v2 (w = 4 dt x u / hbar): dP/dq multiplies the theta-space factor d_k by
// i w_q(k, x).
//
// Precision: the complex type C is float2 (complex64 state, FP32 transforms;
// phase arguments formed and reduced to one turn in FP64, then sincospif) or
// double2 (complex128 state and transforms, sincospi).  Sums are FP64.
// No counterpart in the reference (it has no gradients).
#pragma once
#include "wig_rfft.cuh"
#include "wig_wigner.cuh"

namespace wig {

struct AArgs {
  int n_x, n_p;
  int damped;
  double dt, hbar, mass, dx, dp, dtheta, dlambda;
  double v4, v2, v0;
  double cl1, cl2, cl3;   // imaginary parts of a1, a2, a3
  const void* tw_x;       // register-FFT twiddles of n_x (2 n_x entries of C: forward, inverse)
  const void* tw_p;       // of n_p
  const double* rtab;     // [n_x] exp(-D_lambda lambda^2) / n_x   (per frequency)
  const double* mm;       // [n_x] mask1 mask2 / n_p                (per column)
  const double* rth;      // [n_p] exp(-D_theta theta^2 dt)        (per frequency)
  const double* sfp;      // [n_p] sign(p) f(p)
  const double* ths;      // [n_p] theta / n_p
  double2* pend;          // [1] pending normalisation 1/s of the state (damped forward)
  double2* coef;          // [2] (1/conj(s), -conj(beta)) of the adjoint step being run
};

template <class C> struct CScalar;
template <> struct CScalar<float2> { typedef float T; };
template <> struct CScalar<double2> { typedef double T; };

template <class C> __device__ __forceinline__ C cmk(double x, double y) {
  C r;
  r.x = (typename CScalar<C>::T)x;
  r.y = (typename CScalar<C>::T)y;
  return r;
}

__device__ __forceinline__ int ashift(int k, int n) { return k < n / 2 ? k : k - n; }

// r e^{-2 pi i s t}, t reduced to one turn in FP64 (s = +-1)
template <class C> __device__ __forceinline__ C adj_turn(double t, double r, double s);
template <> __device__ __forceinline__ float2 adj_turn<float2>(double t, double r, double s) {
  const float f = (float)(t - rint(t));
  float sn, cs;
  sincospif(2.f * f, &sn, &cs);
  const float rf = (float)r;
  return make_float2(rf * cs, -(float)s * rf * sn);
}
template <> __device__ __forceinline__ double2 adj_turn<double2>(double t, double r, double s) {
  const double f = t - rint(t);
  double sn, cs;
  sincospi(2. * f, &sn, &cs);
  return make_double2(r * cs, -s * r * sn);
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

// x-pass, one warp per CTA, rf_spw(NX) rows per warp: out = K (s in) (sgn = +1)
// or K^H in (sgn = -1), s = *pend when use_pend, else 1; in and out may alias.
// The spectrum is staged in natural order in the row's exchange region and the
// kinetic factor applied there in a rolled loop (one copy of the factor code).
template <class C, int NX, int NP>
__device__ __forceinline__ void adj_xpass(const AArgs& a, const C* in, C* out, double sgn, int use_pend) {
  typedef RegFft<C, NX> F;
  constexpr int E = F::E, G = F::G, Q = F::Q, SPW = rf_spw(NX);
  constexpr int XS = NX + (G == 8 ? 8 : 0);
  extern __shared__ float2 sma[];
  C* sm = reinterpret_cast<C*>(sma);
  const C* tw = reinterpret_cast<const C*>(a.tw_x);
  const int lane = threadIdx.x & 31, grp = lane / G, g = lane % G;
  const int row = blockIdx.x * SPW + grp;
  WIG_BOUNDS_CHECK("adjoint x-pass row", row, NP);
  const C* src = in + (size_t)row * NX;
  const C s = use_pend ? cmk<C>(a.pend->x, a.pend->y) : cmk<C>(1., 0.);
  C v[E];
#pragma unroll
  for (int m = 0; m < E; ++m) v[m] = use_pend ? cmul(src[g + G * m], s) : src[g + G * m];
  const SlotX<C, PlainSlot> x{sm, PlainSlot{grp * XS}};
  F::fwdx(v, x, tw, g);
  __syncwarp();
#pragma unroll
  for (int e = 0; e < E; ++e) x.put(g * Q + e / G + E * (e % G), v[e]);
  __syncwarp();
  const double cq = a.dt * a.dp * a.dlambda * (double)ashift(row, NP) / (a.mass * 6.283185307179586477);
#pragma unroll 1
  for (int k = g; k < NX; k += G) x.put(k, cmul(x.get(k), adj_turn<C>(cq * (double)ashift(k, NX), __ldg(a.rtab + k), sgn)));
  __syncwarp();
#pragma unroll
  for (int e = 0; e < E; ++e) v[e] = x.get(g * Q + e / G + E * (e % G));
  F::invx(v, x, tw + NX, g);
  C* dst = out + (size_t)row * NX;
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

// Coalesced load / store of a CT x NP tile of columns [col0, col0 + CT) (swizzled tile).
template <class C, int NP, int CT, int NT>
__device__ __forceinline__ void adj_tile_load(C* tile, const C* src, int nx, int col0) {
  for (int e = threadIdx.x; e < CT * NP; e += NT) {
    const int k = e / CT, c = e & (CT - 1);
    WIG_BOUNDS_CHECK("adjoint tile column", col0 + c, nx);
    tile[k * CT + (c ^ tile_sw<CT>(k))] = src[(size_t)k * nx + col0 + c];
  }
}
template <class C, int NP, int CT, int NT>
__device__ __forceinline__ void adj_tile_store(const C* tile, C* dst, int nx, int col0) {
  for (int e = threadIdx.x; e < CT * NP; e += NT) {
    const int k = e / CT, c = e & (CT - 1);
    WIG_BOUNDS_CHECK("adjoint tile column", col0 + c, nx);
    dst[(size_t)k * nx + col0 + c] = tile[k * CT + (c ^ tile_sw<CT>(k))];
  }
}

// D (herm = false) or D^H (herm = true) of one column held by a lane group, in
// registers (natural-order layout in and out), exchanging through x.
template <class C, int NP, class X>
__device__ __forceinline__ void adj_dissipator(const AArgs& a, C (&w)[RegFft<C, NP>::E], const X& x, const C* tw,
                                               int g, bool herm) {
  typedef RegFft<C, NP> F;
  constexpr int E = F::E, G = F::G, Q = F::Q;
  typedef typename CScalar<C>::T T;
  if (!herm) {
#pragma unroll
    for (int m = 0; m < E; ++m) w[m] = cscale(w[m], (T)__ldg(a.sfp + g + G * m));
  }
  F::fwdx(w, x, tw, g);
#pragma unroll
  for (int i = 0; i < Q; ++i)
#pragma unroll
    for (int b = 0; b < G; ++b) w[i * G + b] = cscale(w[i * G + b], (T)__ldg(a.ths + g * Q + i + E * b));
  __syncwarp();
  F::invx(w, x, tw + NP, g);
  if (herm) {
#pragma unroll
    for (int m = 0; m < E; ++m) w[m] = cscale(w[m], (T)__ldg(a.sfp + g + G * m));
  }
}

// Block sum of NV doubles per thread into out[0..NV) (thread 0 writes).
template <int NT, int NV>
__device__ __forceinline__ void adj_block_sum(double (&v)[NV], double* out) {
  __shared__ double red[NT / 32][NV];
#pragma unroll
  for (int q = 0; q < NV; ++q)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_xor_sync(0xffffffffu, v[q], o);
  const int warp = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0)
#pragma unroll
    for (int q = 0; q < NV; ++q) red[warp][q] = v[q];
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < NV; ++q) {
      double s = 0.;
      for (int w = 0; w < NT / 32; ++w) s += red[w][q];
      out[q] = s;
    }
  }
}

// Forward p-pass: out = P(eps) in (undamped) or U = C P(eps) in (damped, and
// this CTA's share of sum U into part[2 blockIdx.x .. + 1]); U_out (may be
// null) receives a copy of the output.  in and out may alias.  Tiles: T0 (the
// columns; after the Moyal pair A's slots), T1 (damped: the dissipator's
// exchange).
template <class C, int NX, int NP, int WARPS>
__device__ __forceinline__ void adj_ppass(const AArgs& a, const C* in, C* out, C* U_out, double eps, double* part) {
  typedef RegFft<C, NP> F;
  typedef typename CScalar<C>::T T;
  constexpr int E = F::E, G = F::G, Q = F::Q, SPW = rf_spw(NP), CT = WARPS * SPW, NT = WARPS * 32;
  extern __shared__ float2 sma[];
  C* t0 = reinterpret_cast<C*>(sma);
  C* t1 = t0 + CT * NP;
  const C* tw = reinterpret_cast<const C*>(a.tw_p);
  const int col0 = blockIdx.x * CT;
  adj_tile_load<C, NP, CT, NT>(t0, in, NX, col0);
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, grp = lane / G, g = lane % G;
  const int c = adj_col<NP, WARPS>(warp, grp);
  const TileSlot<CT> sl{c};
  const SlotX<C, TileSlot<CT>> x0{t0, sl}, x1{t1, sl};
  C w[E];
#pragma unroll
  for (int m = 0; m < E; ++m) w[m] = x0.get(g + G * m);
  F::fwdx(w, x0, tw, g);
  __syncwarp();
#pragma unroll
  for (int e = 0; e < E; ++e) x0.put(g * Q + e / G + E * (e % G), w[e]);
  __syncwarp();
  const int col = col0 + c;
  double al, be;
  moyal_coeffs(a, a.dx * (double)ashift(col, NX), eps, &al, &be);
  const double mm = __ldg(a.mm + col);
#pragma unroll 1
  for (int k = g; k < NP; k += G) {
    const double j = (double)ashift(k, NP);
    x0.put(k, cmul(x0.get(k), adj_turn<C>(j * fma(be, j * j, al), __ldg(a.rth + k) * mm, 1.)));
  }
  __syncwarp();
#pragma unroll
  for (int e = 0; e < E; ++e) w[e] = x0.get(g * Q + e / G + E * (e % G));
  F::invx(w, x0, tw + NP, g);
  if (a.damped) {
    // U = A + a3 D(A + a2 D(A + a1 D A)); A kept in T0's slots, exchange in T1's
    __syncwarp();
#pragma unroll
    for (int m = 0; m < E; ++m) x0.put(g + G * m, w[m]);
#pragma unroll 1
    for (int it = 0; it < 3; ++it) {
      adj_dissipator<C, NP>(a, w, x1, tw, g, false);
      const T ci = (T)(it == 0 ? a.cl1 : (it == 1 ? a.cl2 : a.cl3));
      __syncwarp();
#pragma unroll
      for (int m = 0; m < E; ++m) {
        const C A = x0.get(g + G * m);
        w[m] = cmk<C>(A.x - ci * w[m].y, A.y + ci * w[m].x);
      }
    }
    double su[2] = {0., 0.};
#pragma unroll
    for (int m = 0; m < E; ++m) { su[0] += (double)w[m].x; su[1] += (double)w[m].y; }
    adj_block_sum<NT, 2>(su, part + 2 * blockIdx.x);
  }
  __syncwarp();
#pragma unroll
  for (int m = 0; m < E; ++m) x0.put(g + G * m, w[m]);
  __syncthreads();
  adj_tile_store<C, NP, CT, NT>(t0, out, NX, col0);
  if (U_out) adj_tile_store<C, NP, CT, NT>(t0, U_out, NX, col0);
}

// Adjoint p-pass of step n: lam <- P(eps_n)^H C^H N_n^H lam (damped) or
// P(eps_n)^H lam, and this CTA's shares of dL/d eps_n, dL/dv4 and dL/dv2 into
// part[3 blockIdx.x .. + 2].  N_n^H is the uniform map lam -> coef[0] lam +
// coef[1] (wiga_adj_coef).  Tiles: T0 (lam), T1 (the dissipator's exchange,
// then Y_n).
template <class C, int NX, int NP, int WARPS>
__device__ __forceinline__ void adj_ppass_T(const AArgs& a, C* lam, const C* Y, double eps, double* part) {
  typedef RegFft<C, NP> F;
  typedef typename CScalar<C>::T T;
  constexpr int E = F::E, G = F::G, Q = F::Q, SPW = rf_spw(NP), CT = WARPS * SPW, NT = WARPS * 32;
  extern __shared__ float2 sma[];
  C* t0 = reinterpret_cast<C*>(sma);
  C* t1 = t0 + CT * NP;
  const C* tw = reinterpret_cast<const C*>(a.tw_p);
  const int col0 = blockIdx.x * CT;
  adj_tile_load<C, NP, CT, NT>(t0, lam, NX, col0);
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, grp = lane / G, g = lane % G;
  const int c = adj_col<NP, WARPS>(warp, grp);
  const TileSlot<CT> sl{c};
  const SlotX<C, TileSlot<CT>> x0{t0, sl}, x1{t1, sl};
  C w[E];
  if (a.damped) {
    const C c1 = cmk<C>(a.coef[0].x, a.coef[0].y), c0 = cmk<C>(a.coef[1].x, a.coef[1].y);
#pragma unroll
    for (int m = 0; m < E; ++m) {
      w[m] = cadd(cmul(x0.get(g + G * m), c1), c0);
      x0.put(g + G * m, w[m]);   // mu, the Horner base (each lane rewrites only its own slots)
    }
#pragma unroll 1
    for (int it = 0; it < 3; ++it) {
      adj_dissipator<C, NP>(a, w, x1, tw, g, true);
      const T ci = -(T)(it == 0 ? a.cl1 : (it == 1 ? a.cl2 : a.cl3));   // conj(i c) = -i c
      __syncwarp();
#pragma unroll
      for (int m = 0; m < E; ++m) {
        const C M = x0.get(g + G * m);
        w[m] = cmk<C>(M.x - ci * w[m].y, M.y + ci * w[m].x);
      }
    }
    __syncwarp();
#pragma unroll
    for (int m = 0; m < E; ++m) x0.put(g + G * m, w[m]);   // lam_A
  }
  __syncthreads();   // every group is done with T1 before Y overwrites it
  adj_tile_load<C, NP, CT, NT>(t1, Y, NX, col0);
  __syncthreads();
  // F Y_n, staged in natural order in T1's slots
#pragma unroll
  for (int m = 0; m < E; ++m) w[m] = x1.get(g + G * m);
  F::fwdx(w, x1, tw, g);
  __syncwarp();
#pragma unroll
  for (int e = 0; e < E; ++e) x1.put(g * Q + e / G + E * (e % G), w[e]);
  // F lam_A, staged in natural order in T0's slots
#pragma unroll
  for (int m = 0; m < E; ++m) w[m] = x0.get(g + G * m);
  F::fwdx(w, x0, tw, g);
  __syncwarp();
#pragma unroll
  for (int e = 0; e < E; ++e) x0.put(g * Q + e / G + E * (e % G), w[e]);
  __syncwarp();
  const int col = col0 + c;
  const double xc = a.dx * (double)ashift(col, NX);
  double al, be;
  moyal_coeffs(a, xc, eps, &al, &be);
  const double mm = __ldg(a.mm + col);
  const double h = 0.5 * a.hbar * a.dtheta;   // u = h j
  double gq[3] = {0., 0., 0.};
#pragma unroll 1
  for (int k = g; k < NP; k += G) {
    const double j = (double)ashift(k, NP);
    const C d = adj_turn<C>(j * fma(be, j * j, al), __ldg(a.rth + k) * mm, 1.);
    const C yd = cmul(x1.get(k), d);
    const C U = x0.get(k);
    // Re(i conj(U) yd) = U.y yd.x - U.x yd.y
    const double re = (double)U.y * (double)yd.x - (double)U.x * (double)yd.y;
    const double u = h * j;
    gq[0] += j * re;
    gq[1] += xc * u * (xc * xc + u * u) * re;
    gq[2] += xc * u * re;
    x0.put(k, cmul(U, cconj(d)));
  }
  gq[0] *= a.dt * a.dtheta;
  gq[1] *= 8. * a.dt / a.hbar;
  gq[2] *= 4. * a.dt / a.hbar;
  __syncwarp();
#pragma unroll
  for (int e = 0; e < E; ++e) w[e] = x0.get(g * Q + e / G + E * (e % G));
  F::invx(w, x0, tw + NP, g);
  __syncwarp();
#pragma unroll
  for (int m = 0; m < E; ++m) x0.put(g + G * m, w[m]);
  adj_block_sum<NT, 3>(gq, part + 3 * blockIdx.x);
  __syncthreads();
  adj_tile_store<C, NP, CT, NT>(t0, lam, NX, col0);
}

}  // namespace wig
