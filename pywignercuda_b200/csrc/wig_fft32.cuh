// Warp-level FP32 Stockham FFT for sm_100a.
//
// One warp transforms SPW sequences of length N (power of two) that live in
// shared memory; the warp synchronises with __syncwarp only, so the warps of a
// CTA progress independently.  Radix 16 stages (a 16-point DFT held in
// registers as two radix-4 levels) while N/NS >= 16, then one 8 / 4 / 2 stage.
// Element k of sequence s sits at s*SEQ + k + (k >> 4): one padding slot every
// 16 elements keeps the stride-16 writes of the first stage on distinct banks
// (8-byte accesses are served per half-warp).
//
// Twiddles come from per-stage tables in shared memory: for a stage that
// combines sub-transforms of length NS with radix R, T[(r-1)*NS + k] =
// exp(-2 pi i k r / (NS R)) for r = 1..R-1, k < NS (float, rounded from
// extended precision on the host), so the lanes of a warp (consecutive k) read
// consecutive entries.  stage_tw_offset() gives each stage's offset; a size's
// tables take stage_tw_size(N) entries.  Forward = exp(-i ...), inverse
// unnormalised.
#pragma once
#include "wig_fft.cuh"

namespace wig {

__device__ __forceinline__ int pad16(int k) { return k + (k >> 4); }
__host__ __device__ constexpr int seq_stride32(int n) { return n + (n >> 4); }

template <bool INV> __device__ __forceinline__ void dft16(float2* v) {
  // 16-point DFT as 4 x 4: columns (n = 4a + b) first, then twiddles W16^{b k1}, then rows
  const float c1 = 0.92387953251128675613f, s1 = 0.38268343236508977173f, h = 0.70710678118654752440f;
  float2 t[16];
#pragma unroll
  for (int b = 0; b < 4; ++b) {
    float2 a0 = v[b], a1 = v[b + 4], a2 = v[b + 8], a3 = v[b + 12];
    dft4<INV>(a0, a1, a2, a3);
    t[b] = a0; t[b + 4] = a1; t[b + 8] = a2; t[b + 12] = a3;   // t[4*k1 + b]
  }
  // twiddle W16^{b*k1}, forward W16 = exp(-2 pi i / 16)
  const float sg = INV ? 1.f : -1.f;
  const float2 w1 = make_float2(c1, sg * s1), w2 = make_float2(h, sg * h), w3 = make_float2(s1, sg * c1);
  const float2 w4 = make_float2(0.f, sg * 1.f), w6 = make_float2(-h, sg * h), w9 = make_float2(-c1, -sg * s1);
  t[5] = cmul(t[5], w1);  t[6] = cmul(t[6], w2);  t[7] = cmul(t[7], w3);
  t[9] = cmul(t[9], w2);  t[10] = cmul(t[10], w4); t[11] = cmul(t[11], w6);
  t[13] = cmul(t[13], w3); t[14] = cmul(t[14], w6); t[15] = cmul(t[15], w9);
#pragma unroll
  for (int k1 = 0; k1 < 4; ++k1) {
    float2 a0 = t[4 * k1], a1 = t[4 * k1 + 1], a2 = t[4 * k1 + 2], a3 = t[4 * k1 + 3];
    dft4<INV>(a0, a1, a2, a3);
    v[k1] = a0; v[k1 + 4] = a1; v[k1 + 8] = a2; v[k1 + 12] = a3;   // X[k1 + 4 k2]
  }
}

template <int R, bool INV> __device__ __forceinline__ void dft32(float2* v) {
  if (R == 16) dft16<INV>(v);
  else if (R == 8) dft8<INV>(v);
  else if (R == 4) dft4<INV>(v[0], v[1], v[2], v[3]);
  else dft2<INV>(v[0], v[1]);
}

template <int N, int NS> struct Radix32 {
  static constexpr int rem = N / NS;
  static constexpr int value = rem >= 16 ? 16 : rem;   // 16 or the remaining 8 / 4 / 2
};

__host__ __device__ constexpr int radix32_of(int n, int ns) { return n / ns >= 16 ? 16 : n / ns; }
// entries of the stages before the one that starts at sub-length NS
__host__ __device__ constexpr int stage_tw_offset(int n, int ns) {
  int off = 0;
  for (int s = 1; s < ns; s *= radix32_of(n, s)) off += (s > 1 ? (radix32_of(n, s) - 1) * s : 0);
  return off;
}
__host__ __device__ constexpr int stage_tw_size(int n) { return stage_tw_offset(n, n); }

// One stage over the warp's SPW sequences (s: the warp's first sequence,
// sequences SEQ elements apart).
template <int N, int NS, int SPW, int SEQ, bool INV>
__device__ __forceinline__ void warp_fft_stage(float2* s, const float2* tw, int lane) {
  constexpr int R = Radix32<N, NS>::value;
  constexpr int NBF = N / R;
  constexpr int TOT = SPW * NBF;
  constexpr int PER = (TOT + 31) / 32;
  constexpr int TWO = stage_tw_offset(N, NS);
  float2 v[PER][R];
#pragma unroll
  for (int m = 0; m < PER; ++m) {
    const int q = lane + 32 * m;
    if ((TOT % 32) == 0 || q < TOT) {
      const int sq = q / NBF, j = q % NBF;
#pragma unroll
      for (int r = 0; r < R; ++r) v[m][r] = s[sq * SEQ + pad16(j + r * NBF)];
    }
  }
  __syncwarp();
#pragma unroll
  for (int m = 0; m < PER; ++m) {
    const int q = lane + 32 * m;
    if ((TOT % 32) == 0 || q < TOT) {
      const int sq = q / NBF, j = q % NBF;
      const int k = j & (NS - 1);
      if (NS > 1) {
#pragma unroll
        for (int r = 1; r < R; ++r) {
          float2 w = tw[TWO + (r - 1) * NS + k];
          if (INV) w.y = -w.y;
          v[m][r] = cmul(v[m][r], w);
        }
      }
      dft32<R, INV>(v[m]);
      const int d = (j - k) * R + k;
#pragma unroll
      for (int r = 0; r < R; ++r) s[sq * SEQ + pad16(d + r * NS)] = v[m][r];
    }
  }
  __syncwarp();
}

template <int N, int NS, int SPW, int SEQ, bool INV> struct WarpFft {
  __device__ __forceinline__ static void run(float2* s, const float2* tw, int lane) {
    warp_fft_stage<N, NS, SPW, SEQ, INV>(s, tw, lane);
    WarpFft<N, NS * Radix32<N, NS>::value, SPW, SEQ, INV>::run(s, tw, lane);
  }
};
template <int N, int SPW, int SEQ, bool INV> struct WarpFft<N, N, SPW, SEQ, INV> {
  __device__ __forceinline__ static void run(float2*, const float2*, int) {}
};

// FFT of the warp's SPW sequences, SEQ elements apart (caller has
// __syncwarp'ed; returns synced).  Out of line: each (N, SPW, SEQ, direction)
// is compiled once however many times a kernel calls it, which keeps the
// batched kernels (several size classes, up to ten FFTs each) small enough for
// the instruction cache.
template <int N, int SPW, int SEQ, bool INV>
__device__ __noinline__ void warp_fft_cs(float2* s, const float2* tw, int lane) {
  WarpFft<N, 1, SPW, SEQ, INV>::run(s, tw, lane);
}

template <int N, int SPW, bool INV>
__device__ __forceinline__ void warp_fft(float2* s, const float2* tw, int lane) {
  warp_fft_cs<N, SPW, seq_stride32(N), INV>(s, tw, lane);
}

}  // namespace wig
