// Batched Wigner2D propagation: many independent instances of uneven grid
// sizes advanced together, one x-pass launch and one p-pass launch per step
// over a work list that spans every instance (x-items: blocks of rows, p-items:
// blocks of columns).  Every sequence (a row in the x-pass, a column in the
// p-pass) is transformed by the register-resident FFT of wig_rfft.cuh: rf_g(N)
// lanes of a warp hold its N elements in registers, so the whole p-pass --
// forward FFT, Moyal factor, inverse FFT, the three Caldeira-Leggett dissipator
// applications (six more FFTs), observables -- runs on registers, with shared
// memory only for the coalescing tile and one exchange per FFT.
//
// Storage: W is the real Wigner function, FP32, one float per grid point
// (instance i a row-major (n_p, n_x) block at its offset); two real rows or
// columns share one complex transform.
//
// Precision (WIGB_PREC, one value per compiled batch):
//   0  FP32 transforms and pointwise factors throughout;
//   1  the kinetic (x-pass) and Moyal (p-pass) transform pairs and their
//      factors in FP64; the three dissipator pairs in FP64 on grids of at most
//      WIGB_DISS64_MAXN points along p and in FP32 on larger ones.  The
//      dissipator's contribution is scaled by 2 gamma dt (~1e-3), so its FP32
//      rounding is a small fraction of an FP32 transform's -- except on coarse
//      grids, where theta_max p_max = pi p_max^2 / dp is small and strongly
//      damped instances (gamma ~ 0.2) would otherwise carry ~1e-6 energy
//      error after 2000 steps; those grids are a few percent of a batch's
//      points.  The kinetic and Moyal pairs carry the full state, and their
//      FP32 rounding, spread over the grid and weighted by H(x, p) at its
//      edges, is what drifts the energy in the FP32 form.
// In both, FP64 forms the large phase arguments (dt*lambda*p/m and
// dt*[V(x - hbar theta/2) - V(x + hbar theta/2)]/hbar, the latter from the
// exact polynomial expansion, both in units of 2 pi) and reduces them to one
// turn, and the observables are FP64 (per-column moments, FP64 tree /
// per-instance reductions).
//
// Normalisation (GPU_Wigner2D_FFT.Run :1912-1913): every p-item writes FP64
// partial sums; the last CTA of an instance to finish (arrival counter, no
// waiting) reduces them in item order, writes that step's observables and the
// instance's pending scale, which the next x-pass applies on load.
#pragma once
#include "wig_rfft.cuh"
#include "wig_wigner.cuh"

#ifndef WIGB_WARPS
#define WIGB_WARPS 8
#endif
#ifndef WIGB_PREC
#define WIGB_PREC 0
#endif
#ifndef WIGB_DISS64_MAXN
#define WIGB_DISS64_MAXN 256
#endif
#define WIGB_NT (WIGB_WARPS * 32)

namespace wig {

struct BInst {
  int n_x, n_p;
  int damp;          // 0 none, 1 Caldeira-Leggett
  int ff;            // f(p): 0 |p|, 1 p^2/sqrt(p^2 + f_eps)
  long long off;     // element offset in the packed state buffer
  int xitem0, n_xitems, pitem0, n_pitems;
  int tw_x, tw_p;    // offsets of the instance's twiddle tables (2N entries each) in the table buffer
  int ft_x, ft_p;    // offsets of its float tables: [rtab n_x][mm n_x][gtab 2 n_x] and [rth n_p][sfp n_p][ths n_p]
  int fd_x, fd_p;    // offsets of its double tables: [rtab n_x][mm n_x][gtab 2 n_x] and [rth n_p][sfp n_p][ths n_p]
  double dt, hbar, mass, dx, dp, dtheta, dlambda, D_theta, D_lambda, f_eps;
  double v4, v2, v1, v0;   // V(x) = v4 x^4 + v2 x^2 + v1 x + v0
  double cl_k1, cl_k12, cl_c3;   // imaginary parts of the Caldeira-Leggett Horner coefficients
};

struct BArgs {
  const BInst* inst;
  const int2* xitems;    // (instance, first row)
  const int2* pitems;    // (instance, first column)
  float* W;              // packed real states
  const float2* tw;      // register-FFT twiddles, FP32
  const double2* tw64;   // the same tables in FP64 (same offsets)
  const float* ft;
  const double* fd;
  double* partials;      // [n_pitems][NACC]
  unsigned* counters;    // [n_inst]
  unsigned* tickets;     // [2] work-list tickets of the x- and p-pass (zero between launches)
  double* scale;         // [n_inst] pending normalisation, applied by the next x-pass
  unsigned* status;      // [1] set to 1 by a bounded wait that gave up (read and cleared by the host)
  double* obs;           // [n_inst][obs_stride][NOBS]
  int obs_stride;
  unsigned step;         // the launch's step index (t_index0 + n): the stochastic-rounding key
};

// Shared memory of one item: the x-pass exchange regions and row staging buffer
// (bx_exch, bx_stage), the p-pass tile (float2 units).  The twiddle and factor
// tables are read through the read-only data path (a few KB per size,
// L1-resident).  x-pass: each lane group carries two rows packed into one
// complex sequence and holds, per row pair, the transform exchange / spectrum
// region.
__host__ __device__ constexpr int bx_rows(int n, int warps) { return 2 * warps * rf_spw(n); }
// (the x-pass's shared memory: bx_exch / bx_stage below)
// The p-pass packs two real columns into one complex sequence for the
// Caldeira-Leggett part (see batch_p_item): an item is BP_PACK column groups.
constexpr int BP_PACK = 2;
__host__ __device__ constexpr int bp_cols(int n, int warps) { return BP_PACK * warps * rf_spw(n); }
__host__ __device__ constexpr int bp_smem(int n, int warps) { return BP_PACK * warps * rf_spw(n) * n; }

// p-pass: column of the CT-wide tile owned by group `grp` of warp `warp`.
// With 8-lane groups two sequences share a half-warp; pairing columns c and
// c ^ PM keeps their tile accesses on distinct bank pairs.
template <int N>
__device__ __forceinline__ int rf_col(int warp, int grp) {
  constexpr int G = rf_g(N), SPW = rf_spw(N), CT = WIGB_WARPS * SPW;
  if constexpr (G == 8) {
    constexpr int PM = CT / 2 < 8 ? CT / 2 : 8;
    const int hw = 2 * warp + (grp >> 1);
    const int base = (hw & (PM - 1)) | ((hw / PM) * 2 * PM);
    return base ^ ((grp & 1) * PM);
  } else {
    return warp * SPW + grp;
  }
}

// signed FFT-shifted index of array position k (coordinate = step * index)
__device__ __forceinline__ int shifted(int k, int n) { return k < n / 2 ? k : k - n; }

// e^{-2 pi i t} * r, t reduced to one turn in FP64
__device__ __forceinline__ float2 turn_factor(double t, float r) {
  const float f = (float)(t - rint(t));
  float sn, cs;
  sincospif(2.f * f, &sn, &cs);
  return make_float2(r * cs, -r * sn);
}

// e^{-2 pi i t} * r in FP64, t reduced to one turn
__device__ __forceinline__ double2 turn_factor64(double t, double r) {
  const double f = t - rint(t);
  double sn, cs;
  sincospi(2. * f, &sn, &cs);
  return make_double2(r * cs, -r * sn);
}

// ---------------------------------------------------------- stochastic rounding
// The mixed form (WIGB_PREC 1) computes each pass in FP64 and stores W in FP32.
// Rounding to nearest there loses, at every point whose change over one pass is
// below half an FP32 ulp (the slow rows and columns near the distribution's
// peak, the late approach to a damped equilibrium), that change on every step,
// so the slow part of the dynamics stalls and the energy error grows linearly
// (stagnation: M. Croci and M. B. Giles, "Effects of round-to-nearest and
// stochastic rounding in the numerical solution of the heat equation in low
// precision", IMA J. Numer. Anal. 43 (2023)).  Stochastic rounding -- up with
// probability equal to the remainder's fraction of the ulp -- keeps every change
// in expectation.  Done in the integer domain: 29 random bits (the bits a double
// carries below a float's mantissa) are added to the double's magnitude and the
// result truncated to FP32.  Exact for |v| in the FP32 normal range; below it
// (|v| < 2^-126, nothing there weighs in an observable) the rounding is biased
// toward zero; NaN and infinities stay non-finite.
//
// The random words: each lane seeds a stream by hashing (step, pass, the index
// of its first element), then takes one linear congruential step per element
// (the top 29 bits of the 32-bit state are used).  A run is a function of its
// inputs and t_index0: graph and non-graph runs agree bit for bit.
// sr_mix: the "lowbias32" 32-bit integer hash (C. Wellons, hash-prospector).
__host__ __device__ __forceinline__ unsigned sr_mix(unsigned x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}
// the key of one pass of one step (pass 0: x-pass, 1: p-pass)
__device__ __forceinline__ unsigned sr_key(unsigned step, unsigned pass) { return sr_mix(2u * step + pass + 0x9e3779b9u); }
// the random word of element e (index into the packed state): a stream's seed
__device__ __forceinline__ unsigned sr_word(unsigned key, long long e) {
  return sr_mix((unsigned)e ^ key ^ (0x85ebca6bu * (unsigned)(e >> 32)));
}
// a lane's stream of random words (LCG constants of Numerical Recipes, 2nd ed., 7.1)
struct SrStream {
  unsigned s;
  __device__ __forceinline__ unsigned next() {
    s = s * 1664525u + 1013904223u;
    return s;
  }
};
// v rounded to FP32: stochastically for double, unchanged for float
__device__ __forceinline__ float store_round(double v, unsigned u) {
  return __double2float_rz(__longlong_as_double(__double_as_longlong(v) + (long long)(u >> 3)));
}
__device__ __forceinline__ float store_round(float v, unsigned) { return v; }

struct Kahan {
  double s = 0., c = 0.;
  __device__ __forceinline__ void add(double v) {
    const double y = v - c, t = s + y;
    c = (t - s) - y;
    s = t;
  }
};

__device__ __forceinline__ void accumulate_obs_k(Kahan (&acc)[NACC], float v, double x, double p,
                                                 const BInst& I) {
  const double w = v;
  const double dV = (4. * I.v4 * x * x + 2. * I.v2) * x + I.v1;
  const double V = ((I.v4 * x * x + I.v2) * x + I.v1) * x + I.v0;
  acc[0].add(w);
  acc[2].add(w * x);
  acc[3].add(w * x * x);
  acc[4].add(w * p);
  acc[5].add(w * p * p);
  acc[6].add(w * p * x);
  acc[7].add(w * dV);
  acc[8].add(w * p * dV);
  acc[9].add(w * x * dV);
  acc[10].add(w * (p * p / (2. * I.mass) + V));
  if (w < 0.) acc[11].add(w);
}

// Write this CTA's partials; the last CTA of the instance reduces them (a fixed
// order of Kahan sums), writes the sample's observables and the instance's scale.
// mode: 0 none (scale 1), 1 normalise.
template <int NT>
__device__ __forceinline__ void batch_item_done(const BArgs& A, int inst, const BInst& I, int item,
                                                double (&v)[NACC], int mode, int sample) {
  __shared__ double red[NT / 32][NACC];
  __shared__ int s_last;
  block_sum<NT, NACC>(v, red);
  if (threadIdx.x < NACC) A.partials[(size_t)item * NACC + threadIdx.x] = red[0][threadIdx.x];
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = (atomicAdd(&A.counters[inst], 1u) == (unsigned)(I.n_pitems - 1));
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  // 16 strided Kahan sums per accumulator, combined in a fixed order
  __shared__ double part[NACC][17];
  __shared__ double tot[NACC];
  for (int q = threadIdx.x; q < NACC * 16; q += NT) {
    const int v = q >> 4, j = q & 15;
    Kahan k;
    for (int it = j; it < I.n_pitems; it += 16) k.add(__ldcg(&A.partials[(size_t)(I.pitem0 + it) * NACC + v]));
    part[v][j] = k.s - k.c;
  }
  __syncthreads();
  if (threadIdx.x < NACC) {
    Kahan k;
    for (int j = 0; j < 16; ++j) k.add(part[threadIdx.x][j]);
    tot[threadIdx.x] = k.s - k.c;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const double dXdP = I.dx * I.dp;
    const double s = mode == 1 ? 1. / (tot[0] * dXdP) : 1.;   // W is real: a real sum
    double* o = A.obs + ((size_t)inst * A.obs_stride + sample) * NOBS;
    o[0] = s * tot[0] * dXdP;
    for (int k = 1; k < NOBS; ++k) o[k] = s * (dXdP * tot[k + 1]);
    A.scale[inst] = s;
    A.counters[inst] = 0u;
  }
}

// Next work item of a persistent CTA (dynamic: a CTA that falls behind takes
// fewer items).  The CTA drawing the last of the gridDim.x overflowing tickets
// resets the counter for the next launch.  Every thread returns the item.
__device__ __forceinline__ int next_item(unsigned* ticket, int n_items) {
  __shared__ int s_item;
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned t = atomicAdd(ticket, 1u);
    if (t == (unsigned)n_items + gridDim.x - 1u) *ticket = 0u;
    s_item = (int)t;
  }
  __syncthreads();
  return s_item;
}

// ------------------------------------------------------------------ nyquist_real
// The mirror split below is exact where a factor maps Hermitian spectra to
// Hermitian spectra.  At the Nyquist bin k = N/2 (its own mirror) the
// reference's factors are complex, and the split becomes the real-linear map
// Z -> Z (fa + fb)/2 + conj(Z) (fa - fb)/2, whose gain reaches sqrt(2) when the
// two factors' phases differ: any Nyquist content would then grow every step.
// A real sequence's Nyquist coefficient is real, and the reference's result for
// it, Re IFFT[f A], only sees Re f there, so the split uses Re fa, Re fb at
// k = N/2: the same real result, and a contraction.

// ------------------------------------------------------------------ x-pass
// Item: bx_rows(N) consecutive rows; lane group `pair` carries rows ra = row0 +
// 2 pair and rb = ra + 1 packed into z = W(ra) + i W(rb) (W is real), lane g
// holding elements g + G m.  The kinetic factor differs between the two rows,
// so the spectrum is split with its mirror: for real rows a, b with z = a + i b,
//   Z'(k) = [Z(k) (fa + fb) + conj Z(N - k) (fa - fb)] / 2
// is the spectrum of a' + i b', a' = IFFT[fa FFT a], b' = IFFT[fb FFT b]
// (fa, fb map Hermitian spectra to Hermitian spectra).  Rows ra, rb differ by
// one p step, so fb = fa g(lambda) with g = exp(-i dt dp lambda / m), a table.
// One transform pair per two rows.

// Mirror split of a packed spectrum staged in natural order in the exchange x
// (slots 0..N-1), in place:
//   Z'(k) = Z(k) (fa(k) + fb(k)) + conj Z(N - k) (fa(k) - fb(k))
// (fab(k, &fa, &fb) returns the two sequences' factors with the 1/2 folded in).
// Each lane of the group owns the mirror pairs (q, N - q), q = g, g + G, ...,
// q <= N/2, so no other lane reads a slot it rewrites.  The loop stays rolled:
// one copy of the factor code (the phase reduction and sincospi) per kernel.
template <int N, int G, class C, class X, class Fab>
__device__ __forceinline__ void mirror_split(const X& x, int g, const Fab& fab) {
#pragma unroll 1
  for (int q = g; q <= N / 2; q += G) {
    const int km = (N - q) & (N - 1);
    const C Z = x.get(q), P = x.get(km);
    C fa, fb;
    fab(q, &fa, &fb);
    if (q == N / 2) { fa.y = 0.; fb.y = 0.; }       // Nyquist: see nyquist_real
    const C Zn = cadd(cmul(Z, cadd(fa, fb)), cmul(cconj(P), csub(fa, fb)));
    if (km != q) {
      fab(km, &fa, &fb);
      x.put(km, cadd(cmul(P, cadd(fa, fb)), cmul(cconj(Z), csub(fa, fb))));
    }
    x.put(q, Zn);
  }
}

// The precision of an x-pass: its complex type's twiddle and factor tables.
template <class C> struct XPrec;
template <> struct XPrec<float2> {
  __device__ __forceinline__ static const float2* tw(const BArgs& A, const BInst& I) { return A.tw + I.tw_x; }
  // 0.5 r_lambda(k) exp(-2 pi i t), and the row-pair ratio exp(-i dt dp lambda / m)
  __device__ __forceinline__ static float2 fa(const BArgs& A, const BInst& I, double t, int k) {
    return turn_factor(t, 0.5f * __ldg(A.ft + I.ft_x + k));
  }
  __device__ __forceinline__ static float2 g(const BArgs& A, const BInst& I, int N, int k) {
    const float* gt = A.ft + I.ft_x + 2 * N;
    return make_float2(__ldg(gt + 2 * k), __ldg(gt + 2 * k + 1));
  }
};
template <> struct XPrec<double2> {
  __device__ __forceinline__ static const double2* tw(const BArgs& A, const BInst& I) { return A.tw64 + I.tw_x; }
  __device__ __forceinline__ static double2 fa(const BArgs& A, const BInst& I, double t, int k) {
    return turn_factor64(t, 0.5 * __ldg(A.fd + I.fd_x + k));
  }
  __device__ __forceinline__ static double2 g(const BArgs& A, const BInst& I, int N, int k) {
    return __ldg(reinterpret_cast<const double2*>(A.fd + I.fd_x + 2 * N) + k);
  }
};

// One x-item in the arithmetic of C (float2: FP32; double2: FP64, rounded to
// FP32 once on store).  rows: the item's bx_rows(N) rows of W (in global memory
// or staged in shared memory); after_load() runs once every lane holds its two
// rows in registers (the caller may then reuse the staging buffer).  The
// spectrum is staged in natural order in the pair's exchange region (N
// elements of C) and split there in place.
template <class C, int N, class After>
__device__ __forceinline__ void batch_x_item_t(const BArgs& A, int inst, const BInst& I, int row0, const float* rows,
                                               const After& after_load) {
  typedef RegFft<C, N> F;
  typedef XPrec<C> PR;
  constexpr int E = F::E, G = F::G, Q = F::Q, SPW = rf_spw(N);
  constexpr int XS = N + (G == 8 ? 8 : 0);     // region stride (elements of C)
  extern __shared__ float2 smb[];
  C* X = reinterpret_cast<C*>(smb);
  const C* tf = PR::tw(A, I);
  const C* ti = tf + N;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, grp = lane / G, g = lane % G;
  const int pair = warp * SPW + grp;
  const int ra = row0 + 2 * pair;
  WIG_BOUNDS_CHECK("batched x-pass row", ra + 1, I.n_p);
  const double sc = A.scale[inst];
  const float* Ra = rows + (size_t)(2 * pair) * N;
  const float* Rb = Ra + N;
  C v[E];
#pragma unroll
  for (int m = 0; m < E; ++m) {
    v[m].x = (decltype(v[m].x))((double)Ra[g + G * m] * sc);
    v[m].y = (decltype(v[m].y))((double)Rb[g + G * m] * sc);
  }
  after_load();
  const SlotX<C, PlainSlot> x{X, PlainSlot{pair * XS}};
  F::fwdx(v, x, tf, g);
  __syncwarp();   // the transform's exchange reads are done before the spectrum is staged
#pragma unroll
  for (int e = 0; e < E; ++e) x.put(g * Q + e / G + E * (e % G), v[e]);
  __syncwarp();
  // kinetic factor of row a, exp(-i dt lambda p / m), in turns
  const double cq = I.dt * I.dp * I.dlambda * (double)shifted(ra, I.n_p) / (I.mass * 6.283185307179586477);
  mirror_split<N, G, C>(x, g, [&](int k, C* fa, C* fb) {
    const int lj = k < N / 2 ? k : k - N;
    *fa = PR::fa(A, I, cq * (double)lj, k);
    *fb = cmul(*fa, PR::g(A, I, N, k));
  });
  __syncwarp();
#pragma unroll
  for (int e = 0; e < E; ++e) v[e] = x.get(g * Q + e / G + E * (e % G));
  F::invx(v, x, ti, g);
  float* Wa = A.W + I.off + (size_t)ra * N;
  float* Wb = Wa + N;
  SrStream rs{sr_word(sr_key(A.step, 0), (long long)I.off + (long long)ra * N + g)};
#pragma unroll
  for (int m = 0; m < E; ++m) {
    Wa[g + G * m] = store_round(v[m].x, rs.next());
    Wb[g + G * m] = store_round(v[m].y, rs.next());
  }
}

#if WIGB_PREC == 1
typedef double2 XC;
#else
typedef float2 XC;
#endif

// The x-pass's exchange regions (elements of float2: an FP64 region of N double2
// spans 2 N of them) and staging buffer (floats) of one item of size class N.
__host__ __device__ constexpr int bx_exch(int n, int warps, int prec) {
  return warps * rf_spw(n) * (n + (rf_g(n) == 8 ? 8 : 0)) * (prec == 1 ? 2 : 1);
}
__host__ __device__ constexpr int bx_stage(int n, int warps) { return bx_rows(n, warps) * n; }

// ------------------------------------------------------------------ p-pass
// Item: a tile of CT2 = BP_PACK * WIGB_WARPS * rf_spw(N) columns x N rows, staged
// in shared memory (element (k, c) at k CT2 + (c ^ sw(k))) so that the global
// loads and stores are row segments.  Each lane group owns two columns, c1 and
// c2 = c1 + CT2 / 2, packed into one complex sequence z = Re W(c1) + i Re W(c2)
// (W, the Wigner function, is real):
//   it = 0:     the Moyal pair.  The factor depends on x, so the packed spectrum
//               is split with its mirror (as in the x-pass) and each column's
//               factor applied to its own half;
//   it = 1..3 (damped): Caldeira-Leggett.  The dissipator polynomial
//               z -> A + i c D(z), D(z) = IFFT[theta/N FFT(sign(p) f(p) z)], is
//               complex-linear and the same for every column, so it acts on the
//               two real columns at once.
// The results are Re z, Im z: a damped step costs 4 transform pairs per 2
// columns instead of 8, and the imaginary rounding noise of W (~1e-8 in FP32)
// is dropped.
template <int N>
__device__ __forceinline__ void batch_p_item(const BArgs& A, int inst, const BInst& I, int col0, int item,
                                             int sample) {
  typedef RegFft<float2, N> F;
  constexpr int E = F::E, G = F::G, Q = F::Q, SPW = rf_spw(N), CT = WIGB_WARPS * SPW, CT2 = BP_PACK * CT;
  constexpr int NT = WIGB_NT;
  static_assert(BP_PACK == 2, "two columns per lane group");
  extern __shared__ float2 smb[];
  const float2* tf = A.tw + I.tw_p;
  const float2* ti = tf + N;
  const float* rth = A.ft + I.ft_p;   // exp(-D_theta theta^2 dt)
  const float* sfp = rth + N;         // sign(p) f(p)
  const float* ths = sfp + N;         // theta / N
  float2* tile = smb;                 // after packing, c1's slots hold A (the packed post-Moyal pair)
  const int nx = I.n_x;
  float* Wi = A.W + I.off;
  // coalesced tile load, one register batch per column group (loads in flight
  // before their shared-memory stores)
  constexpr int PER = CT2 * N / NT, LB = PER / BP_PACK;
  static_assert(PER * NT == CT2 * N && PER % LB == 0, "tile load shape");
#pragma unroll 1
  for (int r0 = 0; r0 < PER; r0 += LB) {
    float buf[LB];
#pragma unroll
    for (int r = 0; r < LB; ++r) {
      const int e = threadIdx.x + (r0 + r) * NT;
      WIG_BOUNDS_CHECK("batched p-pass tile column", col0 + (e & (CT2 - 1)), nx);
      WIG_BOUNDS_CHECK("batched p-pass tile row", e / CT2, N);
      buf[r] = Wi[(size_t)(e / CT2) * nx + col0 + (e & (CT2 - 1))];
    }
#pragma unroll
    for (int r = 0; r < LB; ++r) {
      const int e = threadIdx.x + (r0 + r) * NT, k = e / CT2;
      tile[k * CT2 + ((e & (CT2 - 1)) ^ tile_sw<CT2>(k))] = make_float2(buf[r], 0.f);
    }
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, grp = lane / G, g = lane % G;
  const int c1 = rf_col<N>(warp, grp), c2 = c1 + CT;
  const TileSlot<CT2> sl1{c1}, sl2{c2};
  // Moyal factor exp(-i dt [V(x - u) - V(x + u)] / hbar) r_theta mask1 mask2 / N,
  // u = hbar theta / 2 = h j:  V(x - u) - V(x + u) = -2u (a3 + a1 u^2); phase in turns
  const double h = 0.5 * I.hbar * I.dtheta;
  const double kk = -I.dt * h / (3.141592653589793238 * I.hbar);
  const double xa = I.dx * (double)shifted(col0 + c1, nx), xb = I.dx * (double)shifted(col0 + c2, nx);
  const double ala = kk * ((4. * I.v4 * xa * xa + 2. * I.v2) * xa + I.v1);
  const double alb = kk * ((4. * I.v4 * xb * xb + 2. * I.v2) * xb + I.v1);
  const double bea = kk * h * h * (4. * I.v4 * xa), beb = kk * h * h * (4. * I.v4 * xb);
  const float mma = __ldg(A.ft + I.ft_x + nx + col0 + c1), mmb = __ldg(A.ft + I.ft_x + nx + col0 + c2);
  const bool damped = I.damp == 1;
  const int n_it = damped ? 4 : 1;
  float2 w[E];
#if WIGB_PREC == 1
  // FP64 Moyal pair: the packed columns are widened, transformed, split with
  // the spectrum's mirror and multiplied by the FP64 factors in place (the
  // exchange and the staged spectrum use c1's and c2's slots as doubles, PairX),
  // transformed back and rounded to FP32 once; the dissipator pairs below run
  // in FP32 from there.
  constexpr int it0 = 1;
  {
    typedef RegFft<double2, N> F64;
    const double2* tf64 = A.tw64 + I.tw_p;
    const double2* ti64 = tf64 + N;
    const double* rth64 = A.fd + I.fd_p;
    const double mma64 = __ldg(A.fd + I.fd_x + nx + col0 + c1), mmb64 = __ldg(A.fd + I.fd_x + nx + col0 + c2);
    double2 z[E];
#pragma unroll
    for (int m = 0; m < E; ++m) z[m] = make_double2((double)tile[sl1(g + G * m)].x, (double)tile[sl2(g + G * m)].x);
    const PairX<TileSlot<CT2>> px{reinterpret_cast<double*>(tile), sl1, sl2};
    F64::fwdx(z, px, tf64, g);
    __syncwarp();
#pragma unroll
    for (int e = 0; e < E; ++e) px.put(g * Q + e / G + E * (e % G), z[e]);
    __syncwarp();
    mirror_split<N, G, double2>(px, g, [&](int k, double2* fa, double2* fb) {
      const double j = (double)(k < N / 2 ? k : k - N);
      const double r = 0.5 * __ldg(rth64 + k);
      *fa = turn_factor64(j * fma(bea, j * j, ala), r * mma64);
      *fb = turn_factor64(j * fma(beb, j * j, alb), r * mmb64);
    });
    __syncwarp();
#pragma unroll
    for (int e = 0; e < E; ++e) z[e] = px.get(g * Q + e / G + E * (e % G));
    F64::invx(z, px, ti64, g);
    if constexpr (N <= WIGB_DISS64_MAXN) {
      // the dissipator in FP64 as well (coarse grids): A kept in registers, D through PairX
      if (damped) {
        const double* sfp64 = rth64 + N;   // sign(p) f(p)
        const double* ths64 = sfp64 + N;   // theta / N
        double2 A[E];
#pragma unroll
        for (int m = 0; m < E; ++m) A[m] = z[m];
#pragma unroll 1
        for (int it = 0; it < 3; ++it) {
#pragma unroll
          for (int m = 0; m < E; ++m) z[m] = cscale(z[m], __ldg(sfp64 + g + G * m));
          F64::fwdx(z, px, tf64, g);
#pragma unroll
          for (int i = 0; i < Q; ++i)
#pragma unroll
            for (int b = 0; b < G; ++b) z[i * G + b] = cscale(z[i * G + b], __ldg(ths64 + g * Q + i + E * b));
          F64::invx(z, px, ti64, g);
          const double cf = it == 0 ? I.cl_k1 : (it == 1 ? I.cl_k12 : I.cl_c3);
#pragma unroll
          for (int m = 0; m < E; ++m) z[m] = make_double2(A[m].x - cf * z[m].y, A[m].y + cf * z[m].x);
        }
      }
    }
    // rounded to FP32 stochastically (the lane's stream: seeded at its first point of column c1)
    SrStream rs{sr_word(sr_key(A.step, 1), (long long)I.off + (long long)g * nx + col0 + c1)};
#pragma unroll
    for (int m = 0; m < E; ++m) {
      const float a = store_round(z[m].x, rs.next());
      w[m] = make_float2(a, store_round(z[m].y, rs.next()));
    }
  }
  const int n_it_run = N <= WIGB_DISS64_MAXN ? 1 : n_it;
#else
  constexpr int it0 = 0;
  const int n_it_run = n_it;
#pragma unroll
  for (int m = 0; m < E; ++m) {
    const float2 a = tile[sl1(g + G * m)], b = tile[sl2(g + G * m)];
    w[m] = make_float2(a.x, b.x);                  // z = Re W(c1) + i Re W(c2)
  }
#endif
  // One transform pair per pass through this loop (kept rolled so the kernel
  // holds a single copy of each FFT); the exchange runs in c2's slots.
#pragma unroll 1
  for (int it = it0; it < n_it_run; ++it) {
    __syncwarp();   // the previous transform's exchange reads are done before slots change
    if (it == 1) {
#pragma unroll
      for (int m = 0; m < E; ++m) tile[sl1(g + G * m)] = w[m];   // A, the packed post-Moyal pair
    }
    if (it >= 1) {
#pragma unroll
      for (int m = 0; m < E; ++m) w[m] = cscale(w[m], __ldg(sfp + g + G * m));
    }
    F::fwd(w, tile, sl2, tf, g);
    if (it == 0) {
      // the two columns' Moyal factors differ (x), so the packed spectrum is split
      // with its mirror:  Z'(k) = [Z(k) (fa + fb) + conj Z(N - k) (fa - fb)] / 2.
      // The spectrum is staged in natural order in c1's slots, Z' goes through c2's.
      __syncwarp();
#pragma unroll
      for (int e = 0; e < E; ++e) tile[sl1(g * Q + e / G + E * (e % G))] = w[e];
      __syncwarp();
#pragma unroll 2
      for (int e = 0; e < E; ++e) {
        const int i = e / G, b = e % G;
        const int k = g * Q + i + E * b;
        const double j = (double)(b < G / 2 ? k : k - N);
        const float r = __ldg(rth + k);
        float2 fa = turn_factor(j * fma(bea, j * j, ala), r * mma);
        float2 fb = turn_factor(j * fma(beb, j * j, alb), r * mmb);
        if (k == N / 2) { fa.y = 0.f; fb.y = 0.f; }   // Nyquist: see nyquist_real
        const float2 Z = tile[sl1(k)], P = tile[sl1((N - k) & (N - 1))];
        tile[sl2(e * G + g)] = cscale(cadd(cmul(Z, cadd(fa, fb)), cmul(cconj(P), csub(fa, fb))), 0.5f);
      }
      __syncwarp();
#pragma unroll
      for (int e = 0; e < E; ++e) w[e] = tile[sl2(e * G + g)];
    } else {
#pragma unroll
      for (int i = 0; i < Q; ++i)
#pragma unroll
        for (int b = 0; b < G; ++b) w[i * G + b] = cscale(w[i * G + b], __ldg(ths + g * Q + i + E * b));
    }
    F::inv(w, tile, sl2, ti, g);
    if (it >= 1) {
      const float cf = (float)(it == 1 ? I.cl_k1 : (it == 2 ? I.cl_k12 : I.cl_c3));
#pragma unroll
      for (int m = 0; m < E; ++m) {
        const float2 a = tile[sl1(g + G * m)];
        w[m] = make_float2(a.x - cf * w[m].y, a.y + cf * w[m].x);
      }
    }
  }
  // unpack the two real columns: (Re z, 0) -> c1, (Im z, 0) -> c2
  __syncwarp();
#pragma unroll
  for (int m = 0; m < E; ++m) {
    tile[sl1(g + G * m)] = make_float2(w[m].x, 0.f);
    w[m] = make_float2(w[m].y, 0.f);
  }
  __syncwarp();
  // observables: per column, moments sum W, sum W p_j, sum W p_j^2 (FP64), Im and
  // the negative part (FP32 per lane), reduced over the group's lanes
  double acc[NACC];
#pragma unroll
  for (int v = 0; v < NACC; ++v) acc[v] = 0.;
#pragma unroll 1
  for (int q = 0; q < 2; ++q) {
    double s0 = 0., s1 = 0., s2 = 0.;
    float sn = 0.f;
#pragma unroll
    for (int m = 0; m < E; ++m) {
      const float2 v = q == 0 ? tile[sl1(g + G * m)] : w[m];
      const double wr = (double)v.x;
      const double pj = (double)(g + G * m - (m >= E / 2 ? N : 0));
      s0 += wr;
      const double wp = wr * pj;
      s1 += wp;
      s2 = fma(wp, pj, s2);
      sn += fminf(v.x, 0.f);
    }
    double snd = (double)sn;
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) {
      s0 += __shfl_xor_sync(0xffffffffu, s0, o);
      s1 += __shfl_xor_sync(0xffffffffu, s1, o);
      s2 += __shfl_xor_sync(0xffffffffu, s2, o);
      snd += __shfl_xor_sync(0xffffffffu, snd, o);
    }
    if (g == 0) {
      const double x = I.dx * (double)shifted(col0 + (q == 0 ? c1 : c2), nx);
      const double dV = (4. * I.v4 * x * x + 2. * I.v2) * x + I.v1;
      const double V = ((I.v4 * x * x + I.v2) * x + I.v1) * x + I.v0;
      const double M1 = s1 * I.dp, M2 = s2 * (I.dp * I.dp);
      acc[0] += s0;
      acc[2] += s0 * x;
      acc[3] += s0 * x * x;
      acc[4] += M1;
      acc[5] += M2;
      acc[6] += M1 * x;
      acc[7] += s0 * dV;
      acc[8] += M1 * dV;
      acc[9] += s0 * x * dV;
      acc[10] += M2 / (2. * I.mass) + s0 * V;
      acc[11] += snd;
    }
  }
  __syncwarp();
#pragma unroll
  for (int m = 0; m < E; ++m) tile[sl2(g + G * m)] = w[m];
  __syncthreads();
#pragma unroll 8
  for (int r = 0; r < PER; ++r) {
    const int e = threadIdx.x + r * NT, k = e / CT2, cc = e & (CT2 - 1);
    WIG_BOUNDS_CHECK("batched p-pass store column", col0 + cc, nx);
    Wi[(size_t)k * nx + col0 + cc] = tile[k * CT2 + (cc ^ tile_sw<CT2>(k))].x;
  }
  batch_item_done<NT>(A, inst, I, item, acc, I.damp ? 1 : 0, sample);
}

// Initial normalisation and sample 0 (Run :1778-1780), over the p-items.
template <int N>
__device__ __forceinline__ void batch_reduce_item(const BArgs& A, int inst, const BInst& I, int col0, int item,
                                                  int mode, int sample) {
  constexpr int CPB = bp_cols(N, WIGB_WARPS);
  constexpr int NT = WIGB_NT;
  const int nx = I.n_x;
  const float* Wi = A.W + I.off;
  Kahan acc[NACC];
  for (int e = threadIdx.x; e < CPB * N; e += NT) {
    const int k = e / CPB, c = e - k * CPB;
    const int col = col0 + c;
    WIG_BOUNDS_CHECK("batched reduce column", col, nx);
    accumulate_obs_k(acc, Wi[(size_t)k * nx + col], I.dx * shifted(col, nx), I.dp * shifted(k, N), I);
  }
  double v[NACC];
#pragma unroll
  for (int k = 0; k < NACC; ++k) v[k] = acc[k].s + (-acc[k].c);
  batch_item_done<NT>(A, inst, I, item, v, mode, sample);
}

template <int N>
__device__ __forceinline__ void batch_scale_item(const BArgs& A, int inst, const BInst& I, int col0) {
  constexpr int CPB = bp_cols(N, WIGB_WARPS);
  constexpr int NT = WIGB_NT;
  const float sc = (float)A.scale[inst];
  float* Wi = A.W + I.off;
  for (int e = threadIdx.x; e < CPB * N; e += NT) {
    const int k = e / CPB, c = e - k * CPB;
    const size_t g = (size_t)k * I.n_x + col0 + c;
    Wi[g] *= sc;
  }
}

}  // namespace wig
