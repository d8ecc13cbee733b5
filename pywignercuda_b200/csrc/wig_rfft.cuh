// Register-resident FFT for sm_100a (float2 or double2).
//
// A length-N transform (N = E * G, powers of two) is done by a group of G
// lanes of one warp, each lane holding E elements in registers; a warp runs
// 32 / G such sequences side by side.  Write n = g + G m, k = a + E b
// (g, b < G; m, a < E).  Then
//
//   X[a + E b] = sum_g W_G^{g b} W_N^{g a} sum_m x[g + G m] W_E^{m a}
//
// so the forward transform is: an E-point DFT in each lane's registers, the
// twiddles W_N^{g a}, one exchange through shared memory (lane g writes its E
// values, lane t reads back the Q = E / G rows a = t Q + i for all g) and Q
// G-point DFTs in registers.  Every lane's arithmetic is on registers; the
// only shared-memory traffic is one store and one load per element.
//
// Layouts.  Forward input: lane g holds v[m] = x[g + G m] (natural order,
// stride G).  Forward output: lane t holds v[i G + b] = X[t Q + i + E b].  The
// inverse transform takes exactly that layout and returns natural order, so a
// pointwise factor can be applied between them without any reordering.
// Inverse unnormalised (callers fold 1/N into a pointwise factor, exact for a
// power of two).
//
// Exchange slot of (a, g): a G + (g ^ ((a / Q) mod G)).  The XOR spreads both
// the writes (fixed a, consecutive g) and the reads (fixed g, consecutive t)
// over distinct 8-byte bank pairs; the caller maps the N slot numbers of a
// sequence to shared-memory addresses (a functor), so a sequence can use its
// own tile storage as exchange scratch.
//
// Twiddle tables (2N entries per size, host-computed in extended precision,
// read with __ldg: small enough to stay in L1):
//   forward  tf[a G + g]           = W_N^{g a}
//   inverse  ti[(i G + b) G + t]   = W_N^{b (t Q + i)}   (conjugated when used)
// so the lanes of a warp read consecutive entries (or the same entry).
#pragma once
#include "wig_fft.cuh"

namespace wig {

// Elements per lane and lanes per sequence for N in [64, 1024].
__host__ __device__ constexpr int rf_e(int n) { return n >= 512 ? 32 : (n >= 128 ? 16 : 8); }
__host__ __device__ constexpr int rf_g(int n) { return n / rf_e(n); }
__host__ __device__ constexpr int rf_spw(int n) { return 32 / rf_g(n); }   // sequences per warp

// cos(pi j / 16) for any integer j
__host__ __device__ constexpr double cospi16(int j) {
  j = ((j % 32) + 32) % 32;
  if (j > 16) j = 32 - j;
  const bool neg = j > 8;
  if (neg) j = 16 - j;
  double c = 0.;
  switch (j) {
    case 0: c = 1.; break;
    case 1: c = 0.98078528040323044912618223613424; break;
    case 2: c = 0.92387953251128675612818318939679; break;
    case 3: c = 0.83146961230254523707878837761791; break;
    case 4: c = 0.70710678118654752440084436210485; break;
    case 5: c = 0.55557023301960222474283081394853; break;
    case 6: c = 0.38268343236508977172845998403040; break;
    case 7: c = 0.19509032201612826784828486847702; break;
    default: c = 0.; break;
  }
  return neg ? -c : c;
}

// u * c for a compile-time constant c.  In FP32 the constant is applied as a
// compensated pair hi + lo (hi = c rounded, lo = the rounding error), so the
// product carries only the rounding of the arithmetic: a constant rounded to
// float alone has |w|^2 != 1 by up to 6e-8, and a forward/inverse pair of FFTs
// would then scale some spectral components by a fixed factor every step.
__device__ __forceinline__ float mulk(float u, double c) {
  const float hi = (float)c, lo = (float)(c - (double)hi);
  return fmaf(u, hi, u * lo);
}
__device__ __forceinline__ double mulk(double u, double c) { return u * c; }
// u * c + v * s (c, s compile-time constants)
__device__ __forceinline__ float mulk2(float u, double c, float v, double s) {
  const float ch = (float)c, cl = (float)(c - (double)ch), sh = (float)s, sl = (float)(s - (double)sh);
  return fmaf(u, ch, fmaf(v, sh, fmaf(u, cl, v * sl)));
}
__device__ __forceinline__ double mulk2(double u, double c, double v, double s) { return fma(u, c, v * s); }

// v * W_32^j, W_32 = exp(-2 pi i / 32) (forward) or its conjugate (inverse);
// j is a compile-time constant after unrolling.
template <bool INV, class C>
__device__ __forceinline__ C twc32(C v, int j) {
  j &= 31;
  if (j == 0) return v;
  if (j == 16) { v.x = -v.x; v.y = -v.y; return v; }
  if (j == 8) return mul_mi<INV>(v);
  if (j == 24) return mul_mi<!INV>(v);
  const double c = cospi16(j), s = cospi16(8 - j);   // cos, sin of 2 pi j / 32
  C r;
  if ((j & 7) == 4) {   // |c| = |s| = sqrt(1/2): one product per component
    const double h = 0.70710678118654752440084436210485;
    const auto cx = c > 0. ? v.x : -v.x, cy = c > 0. ? v.y : -v.y;   // v c / h
    const auto sx = s > 0. ? v.x : -v.x, sy = s > 0. ? v.y : -v.y;   // v s / h
    if (INV) { r.x = mulk(cx - sy, h); r.y = mulk(sx + cy, h); }
    else     { r.x = mulk(cx + sy, h); r.y = mulk(cy - sx, h); }
    return r;
  }
  if (INV) { r.x = mulk2(v.x, c, v.y, -s); r.y = mulk2(v.x, s, v.y, c); }
  else     { r.x = mulk2(v.x, c, v.y, s);  r.y = mulk2(v.y, c, v.x, -s); }
  return r;
}

// 8-point DFT (radix-2 over two 4-point DFTs), constants through twc32.
template <bool INV, class C> __device__ __forceinline__ void dft8c(C* v) {
  C a[4], b[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) { a[k] = cadd(v[k], v[k + 4]); b[k] = csub(v[k], v[k + 4]); }
  b[1] = twc32<INV>(b[1], 4);
  b[2] = mul_mi<INV>(b[2]);
  b[3] = twc32<INV>(b[3], 12);
  dft4<INV>(a[0], a[1], a[2], a[3]);
  dft4<INV>(b[0], b[1], b[2], b[3]);
#pragma unroll
  for (int m = 0; m < 4; ++m) { v[2 * m] = a[m]; v[2 * m + 1] = b[m]; }
}

// 16-point DFT as 4 x 4 (n = 4 a + b): radix-4 over a, twiddles W_16^{b k1},
// radix-4 over b.  Natural order in and out.
template <bool INV, class C> __device__ __forceinline__ void dft16(C* v) {
  C t[16];
#pragma unroll
  for (int b = 0; b < 4; ++b) {
    C a0 = v[b], a1 = v[b + 4], a2 = v[b + 8], a3 = v[b + 12];
    dft4<INV>(a0, a1, a2, a3);
    t[b] = a0; t[b + 4] = a1; t[b + 8] = a2; t[b + 12] = a3;   // t[4 k1 + b]
  }
#pragma unroll
  for (int k1 = 1; k1 < 4; ++k1)
#pragma unroll
    for (int b = 1; b < 4; ++b) t[4 * k1 + b] = twc32<INV>(t[4 * k1 + b], 2 * b * k1);
#pragma unroll
  for (int k1 = 0; k1 < 4; ++k1) {
    C a0 = t[4 * k1], a1 = t[4 * k1 + 1], a2 = t[4 * k1 + 2], a3 = t[4 * k1 + 3];
    dft4<INV>(a0, a1, a2, a3);
    v[k1] = a0; v[k1 + 4] = a1; v[k1 + 8] = a2; v[k1 + 12] = a3;   // X[k1 + 4 k2]
  }
}

// 32-point DFT: radix-2 decimation in time over two 16-point DFTs.
template <bool INV, class C> __device__ __forceinline__ void dft32(C* v) {
  C e[16], o[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) { e[k] = v[2 * k]; o[k] = v[2 * k + 1]; }
  dft16<INV>(e);
  dft16<INV>(o);
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    const C t = twc32<INV>(o[k], k);
    v[k] = cadd(e[k], t);
    v[k + 16] = csub(e[k], t);
  }
}

template <int R, bool INV, class C> __device__ __forceinline__ void dft_r(C* v) {
  if constexpr (R == 32) dft32<INV>(v);
  else if constexpr (R == 16) dft16<INV>(v);
  else if constexpr (R == 8) dft8c<INV>(v);
  else if constexpr (R == 4) dft4<INV>(v[0], v[1], v[2], v[3]);
  else if constexpr (R == 2) dft2<INV>(v[0], v[1]);
}

template <class C, int N> struct RegFft {
  static constexpr int E = rf_e(N), G = rf_g(N), Q = E / G;
  static_assert(E * G == N && E >= G && (N & (N - 1)) == 0, "RegFft: N must be a power of two in [64, 1024]");

  // lane g (0 <= g < G) of its group; slot(s) maps the sequence's slot s < N to
  // a shared-memory index.
  template <class Slot>
  __device__ __forceinline__ static void fwd(C (&v)[E], C* sm, const Slot& slot, const C* tf, int g) {
    dft_r<E, false>(v);
#pragma unroll
    for (int a = 1; a < E; ++a) v[a] = cmul(v[a], __ldg(tf + a * G + g));
    __syncwarp();
#pragma unroll
    for (int a = 0; a < E; ++a) sm[slot(a * G + (g ^ ((a / Q) & (G - 1))))] = v[a];
    __syncwarp();
#pragma unroll
    for (int i = 0; i < Q; ++i)
#pragma unroll
      for (int b = 0; b < G; ++b) v[i * G + b] = sm[slot((g * Q + i) * G + (b ^ g))];
#pragma unroll
    for (int i = 0; i < Q; ++i) dft_r<G, false>(&v[i * G]);
  }

  template <class Slot>
  __device__ __forceinline__ static void inv(C (&v)[E], C* sm, const Slot& slot, const C* ti, int g) {
#pragma unroll
    for (int i = 0; i < Q; ++i) dft_r<G, true>(&v[i * G]);
#pragma unroll
    for (int i = 0; i < Q; ++i)
#pragma unroll
      for (int b = 0; b < G; ++b)
        if (i > 0 || b > 0) v[i * G + b] = cmul(v[i * G + b], cconj(__ldg(ti + (i * G + b) * G + g)));
    __syncwarp();
#pragma unroll
    for (int i = 0; i < Q; ++i)
#pragma unroll
      for (int b = 0; b < G; ++b) sm[slot((g * Q + i) * G + (b ^ g))] = v[i * G + b];
    __syncwarp();
#pragma unroll
    for (int a = 0; a < E; ++a) v[a] = sm[slot(a * G + (g ^ ((a / Q) & (G - 1))))];
    dft_r<E, true>(v);
  }

  // frequency index of element (i, b) of lane t after fwd
  __device__ __forceinline__ static int kfreq(int t, int i, int b) { return t * Q + i + E * b; }
};

// Slot maps: a plain per-sequence region, or column c of a swizzled row-major
// tile of CT columns (element (k, c) at k CT + (c ^ sw(k))).
struct PlainSlot {
  int base;
  __device__ __forceinline__ int operator()(int s) const { return base + s; }
};

template <int CT>
__host__ __device__ constexpr int tile_sw(int k) { return CT >= 16 ? (k & 15) : ((k / (16 / CT)) & (CT - 1)); }

template <int CT> struct TileSlot {
  int c;
  __device__ __forceinline__ int operator()(int k) const { return k * CT + (c ^ tile_sw<CT>(k)); }
};

}  // namespace wig
