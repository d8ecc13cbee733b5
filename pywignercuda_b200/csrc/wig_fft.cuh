// Shared-memory batched Stockham FFT for sm_100a (double and float).
//
// One CTA transforms NB independent sequences of length N (power of two) that
// live in shared memory.  The element layout is a template functor ("Map") so
// that the same code serves contiguous rows (x-pass: sequence = one grid row)
// and interleaved column tiles (p-pass: sequence = one grid column, the tile
// stored row-major, so element k of column c sits at k*NB + c).
//
// Stockham autosort, mixed radix 16/8/4/2: stage s combines R sub-transforms of
// length Ns into length Ns*R.  Butterfly j (0 <= j < N/R) reads elements
// j + r*N/R, applies twiddles W_{Ns R}^{(j mod Ns) r}, does an R-point DFT and
// writes to (j/Ns)*Ns*R + (j mod Ns) + r*Ns.  Output is in natural order.
// Each stage is done in place through registers: every thread loads all of
// its butterflies' inputs, the CTA synchronises, then every thread writes.
//
// Twiddles come from a table tw[m] = exp(-2 pi i m / N), m < N, computed on
// the host in extended precision; the inverse transform uses the conjugates.
// Forward = exp(-i ...), inverse unnormalised (the callers fold 1/N into a
// pointwise factor, which is exact because N is a power of two).
#pragma once

// WIG_BOUNDS_CHECK(what, i, n): 0 <= i < n.  Compiled in only when WIG_BOUNDS is
// defined, which only the host execution of this device code does (its shim
// provides wig_bounds_fail, which reports and aborts); the kernels the library
// compiles for the GPU carry no such checks and never trap.
#ifdef WIG_BOUNDS
#define WIG_BOUNDS_CHECK(what, i, n)                                                   \
  do {                                                                                 \
    if ((long long)(i) < 0 || (long long)(i) >= (long long)(n)) wig_bounds_fail(what, (long long)(i), (long long)(n)); \
  } while (0)
#else
#define WIG_BOUNDS_CHECK(what, i, n) \
  do {                               \
  } while (0)
#endif

namespace wig {

template <class T> struct V2;
template <> struct V2<double> { typedef double2 t; };
template <> struct V2<float>  { typedef float2 t;  };

__device__ __forceinline__ double2 mk(double a, double b) { return make_double2(a, b); }
__device__ __forceinline__ float2  mk(float a, float b)   { return make_float2(a, b); }

template <class C> __device__ __forceinline__ C cadd(C a, C b) { C r; r.x = a.x + b.x; r.y = a.y + b.y; return r; }
template <class C> __device__ __forceinline__ C csub(C a, C b) { C r; r.x = a.x - b.x; r.y = a.y - b.y; return r; }
// (a.x + i a.y)(b.x + i b.y), the textbook formula (same as pycuda::complex)
template <class C> __device__ __forceinline__ C cmul(C a, C b) {
  C r; r.x = a.x * b.x - a.y * b.y; r.y = a.x * b.y + a.y * b.x; return r;
}
template <class C> __device__ __forceinline__ C cconj(C a) { a.y = -a.y; return a; }
template <class C, class T> __device__ __forceinline__ C cscale(C a, T s) { a.x *= s; a.y *= s; return a; }
// multiply by -i (forward) or +i (inverse)
template <bool INV, class C> __device__ __forceinline__ C mul_mi(C a) {
  C r;
  if (INV) { r.x = -a.y; r.y = a.x; } else { r.x = a.y; r.y = -a.x; }
  return r;
}

// ---------------------------------------------------------------- R-point DFTs
template <bool INV, class C> __device__ __forceinline__ void dft2(C& a, C& b) {
  C t = a; a = cadd(t, b); b = csub(t, b);
}

template <bool INV, class C> __device__ __forceinline__ void dft4(C& v0, C& v1, C& v2, C& v3) {
  C a0 = cadd(v0, v2), a1 = csub(v0, v2), a2 = cadd(v1, v3), a3 = mul_mi<INV>(csub(v1, v3));
  v0 = cadd(a0, a2); v2 = csub(a0, a2); v1 = cadd(a1, a3); v3 = csub(a1, a3);
}

template <bool INV, class C> __device__ __forceinline__ void dft8(C* v) {
  typedef decltype(v[0].x) T;
  const T h = (T)0.70710678118654752440084436210485;   // sqrt(1/2)
  C a[4], b[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) { a[k] = cadd(v[k], v[k + 4]); b[k] = csub(v[k], v[k + 4]); }
  // b_k *= W8^k  (W8 = exp(-+ 2 pi i / 8))
  {
    C t = b[1];
    if (INV) { b[1].x = h * (t.x - t.y); b[1].y = h * (t.x + t.y); }
    else     { b[1].x = h * (t.x + t.y); b[1].y = h * (t.y - t.x); }
    b[2] = mul_mi<INV>(b[2]);
    t = b[3];
    if (INV) { b[3].x = -h * (t.x + t.y); b[3].y = h * (t.x - t.y); }
    else     { b[3].x = h * (t.y - t.x); b[3].y = -h * (t.x + t.y); }
  }
  dft4<INV>(a[0], a[1], a[2], a[3]);
  dft4<INV>(b[0], b[1], b[2], b[3]);
#pragma unroll
  for (int m = 0; m < 4; ++m) { v[2 * m] = a[m]; v[2 * m + 1] = b[m]; }
}

// ---------------------------------------------------------------- radix-8/16/32 kernels
// (also the per-lane DFTs of the register FFT, wig_rfft.cuh)
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

template <int R, bool INV, class C> __device__ __forceinline__ void dft(C* v) {
  if constexpr (R == 2) dft2<INV>(v[0], v[1]);
  else if constexpr (R == 4) dft4<INV>(v[0], v[1], v[2], v[3]);
  else if constexpr (R == 8) dft8<INV>(v);
  else dft16<INV>(v);
}

// ---------------------------------------------------------------- layouts
// Shared-memory layouts.  Both are a linear order plus one padding slot every
// 8 elements (phys = lin + lin/8), which spreads the stride-R accesses of the
// first Stockham stage over distinct 16-byte bank groups.
__device__ __forceinline__ int pad8(int lin) { return lin + (lin >> 3); }
__host__ __device__ constexpr int padded_size(int n) { return n + (n >> 3); }

// Contiguous rows: sequence b, element k at lin = b*N + k; consecutive
// butterflies walk along a row.
template <int N> struct RowMap {
  __device__ __forceinline__ static int idx(int b, int k) { return pad8(b * N + k); }
  template <int NBF> __device__ __forceinline__ static void split(int q, int& b, int& j) { b = q / NBF; j = q % NBF; }
};

// Column tile stored row-major: sequence (column) b, element k at lin = k*NB + b;
// consecutive butterflies walk across the columns first.
template <int NB> struct ColMap {
  __device__ __forceinline__ static int idx(int b, int k) { return pad8(k * NB + b); }
  template <int NBF> __device__ __forceinline__ static void split(int q, int& b, int& j) { b = q % NB; j = q / NB; }
};

// Largest radix <= MAXR that fits the remaining length.  MAXR = 16 takes fewer
// shared-memory round trips (256 = 16 16, 1024 = 16 16 4) but needs about twice the
// registers of MAXR = 8, so it is a per-call-site choice.
template <int N, int NS, int MAXR = 8> struct Radix {
  static constexpr int rem = N / NS;
  static constexpr int value = (MAXR >= 16 && rem >= 16) ? 16 : (rem >= 8 ? 8 : (rem >= 4 ? 4 : 2));
};

// One Stockham stage over all NB sequences.  Phase 1 reads each butterfly's R
// inputs from shared memory and its R-1 twiddles from the (L1-resident) table,
// so the twiddle latency overlaps the barrier; phase 2 computes and writes.
template <class C, int N, int NS, int NB, int NT, bool INV, class Map, int MAXR = 8>
__device__ __forceinline__ void fft_stage(C* s, const C* __restrict__ tw) {
  constexpr int R = Radix<N, NS, MAXR>::value;
  constexpr int NBF = N / R;                 // butterflies per sequence
  constexpr int TOT = NB * NBF;              // butterflies per stage
  constexpr int PER = (TOT + NT - 1) / NT;   // per thread
  constexpr int TWS = N / (NS * R);          // twiddle-table stride of this stage
  const int tid = threadIdx.x;
  C v[PER][R];
  C w[PER][R > 1 ? R - 1 : 1];
#pragma unroll
  for (int m = 0; m < PER; ++m) {
    const int q = tid + m * NT;
    if ((TOT % NT) == 0 || q < TOT) {
      int b, j;
      Map::template split<NBF>(q, b, j);
#pragma unroll
      for (int r = 0; r < R; ++r) v[m][r] = s[Map::idx(b, j + r * NBF)];
      if (NS > 1) {
        const int k = j & (NS - 1);
#pragma unroll
        for (int r = 1; r < R; ++r) w[m][r - 1] = __ldg(&tw[(k * r) * TWS]);
      }
    }
  }
  __syncthreads();
#pragma unroll
  for (int m = 0; m < PER; ++m) {
    const int q = tid + m * NT;
    if ((TOT % NT) == 0 || q < TOT) {
      int b, j;
      Map::template split<NBF>(q, b, j);
      const int k = j & (NS - 1);
      if (NS > 1) {
#pragma unroll
        for (int r = 1; r < R; ++r) v[m][r] = cmul(v[m][r], INV ? cconj(w[m][r - 1]) : w[m][r - 1]);
      }
      dft<R, INV>(v[m]);
      const int d = (j - k) * R + k;
#pragma unroll
      for (int r = 0; r < R; ++r) s[Map::idx(b, d + r * NS)] = v[m][r];
    }
  }
  __syncthreads();
}

template <class C, int N, int NS, int NB, int NT, bool INV, class Map, int MAXR> struct FftRun {
  __device__ __forceinline__ static void run(C* s, const C* __restrict__ tw) {
    fft_stage<C, N, NS, NB, NT, INV, Map, MAXR>(s, tw);
    FftRun<C, N, NS * Radix<N, NS, MAXR>::value, NB, NT, INV, Map, MAXR>::run(s, tw);
  }
};
template <class C, int N, int NB, int NT, bool INV, class Map, int MAXR> struct FftRun<C, N, N, NB, NT, INV, Map, MAXR> {
  __device__ __forceinline__ static void run(C*, const C* __restrict__) {}
};

// Batched FFT of NB sequences of length N in shared memory (caller has
// synchronised before; the CTA is synchronised on return).
template <class C, int N, int NB, int NT, bool INV, class Map, int MAXR = 8>
__device__ __forceinline__ void cta_fft(C* s, const C* __restrict__ tw) {
  FftRun<C, N, 1, NB, NT, INV, Map, MAXR>::run(s, tw);
}

}  // namespace wig
