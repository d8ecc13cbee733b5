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

template <class C, int N> struct RegFft {
  static constexpr int E = rf_e(N), G = rf_g(N), Q = E / G;
  static_assert(E * G == N && E >= G && (N & (N - 1)) == 0, "RegFft: N must be a power of two in [64, 1024]");

  // lane g (0 <= g < G) of its group; x.put(s, v) / x.get(s) store and load
  // the sequence's exchange slot s < N (an exchange functor, see SlotX / PairX).
  template <class X>
  __device__ __forceinline__ static void fwdx(C (&v)[E], const X& x, const C* tf, int g) {
    dft_r<E, false>(v);
#pragma unroll
    for (int a = 1; a < E; ++a) v[a] = cmul(v[a], __ldg(tf + a * G + g));
    __syncwarp();
#pragma unroll
    for (int a = 0; a < E; ++a) x.put(a * G + (g ^ ((a / Q) & (G - 1))), v[a]);
    __syncwarp();
#pragma unroll
    for (int i = 0; i < Q; ++i)
#pragma unroll
      for (int b = 0; b < G; ++b) v[i * G + b] = x.get((g * Q + i) * G + (b ^ g));
#pragma unroll
    for (int i = 0; i < Q; ++i) dft_r<G, false>(&v[i * G]);
  }

  template <class X>
  __device__ __forceinline__ static void invx(C (&v)[E], const X& x, const C* ti, int g) {
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
      for (int b = 0; b < G; ++b) x.put((g * Q + i) * G + (b ^ g), v[i * G + b]);
    __syncwarp();
#pragma unroll
    for (int a = 0; a < E; ++a) v[a] = x.get(a * G + (g ^ ((a / Q) & (G - 1))));
    dft_r<E, true>(v);
  }

  // slot(s) maps the sequence's slot s < N to an index of sm (same element type)
  template <class Slot>
  __device__ __forceinline__ static void fwd(C (&v)[E], C* sm, const Slot& slot, const C* tf, int g);
  template <class Slot>
  __device__ __forceinline__ static void inv(C (&v)[E], C* sm, const Slot& slot, const C* ti, int g);

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

// Exchange functors of RegFft::fwdx / invx.
// SlotX: element s at sm[slot(s)] (the element type of the transform).
template <class C, class Slot> struct SlotX {
  C* sm;
  Slot slot;
  __device__ __forceinline__ void put(int s, C v) const { sm[slot(s)] = v; }
  __device__ __forceinline__ C get(int s) const { return sm[slot(s)]; }
};
// PairX: an FP64 sequence exchanged through the 8-byte slots of two columns of
// a float2 tile: the real part of element s in slot s of column 1, the
// imaginary part in slot s of column 2 (each slot reinterpreted as one double).
template <class Slot> struct PairX {
  double* sm;
  Slot s1, s2;
  __device__ __forceinline__ void put(int s, double2 v) const { sm[s1(s)] = v.x; sm[s2(s)] = v.y; }
  __device__ __forceinline__ double2 get(int s) const { return make_double2(sm[s1(s)], sm[s2(s)]); }
};

template <class C, int N>
template <class Slot>
__device__ __forceinline__ void RegFft<C, N>::fwd(C (&v)[E], C* sm, const Slot& slot, const C* tf, int g) {
  fwdx(v, SlotX<C, Slot>{sm, slot}, tf, g);
}
template <class C, int N>
template <class Slot>
__device__ __forceinline__ void RegFft<C, N>::inv(C (&v)[E], C* sm, const Slot& slot, const C* ti, int g) {
  invx(v, SlotX<C, Slot>{sm, slot}, ti, g);
}

}  // namespace wig
