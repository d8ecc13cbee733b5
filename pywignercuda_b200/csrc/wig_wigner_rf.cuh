// Complex128 Wigner2D passes of the Lie step on the register-resident FFT
// (wig_rfft.cuh), for grids of 64 to 1024 points per axis: the same pointwise
// arithmetic as xpass_body / ppass_body (wig_wigner.cuh) -- the '%f' kernel
// constants, the user's expression strings, sincos of the full phase and the
// reference's operation order -- with each row or column transformed by the
// G lanes of a warp group holding its N elements in registers (one shared-
// memory exchange per transform instead of one round trip per Stockham
// stage, and no CTA-wide barrier inside a transform).
//
// Layout in shared memory.  x-pass: one exchange region per row.  p-pass: a
// row-major tile of C columns in the swizzled layout of a 2-D tensor copy (A,
// the columns and, damped, the base of the Horner form; loaded by TMA with
// WIG_TMA) and, damped, a second tile (B, the dissipator's exchange).
// Pointwise factors are applied to the spectrum staged in natural order in the
// sequence's own slots, in a rolled loop over the frequencies a lane owns, so
// each factor's code (the expression strings, sincos) appears once per kernel.
#pragma once
#include "wig_rfft.cuh"
#include "wig_wigner.cuh"

namespace wig {

// ---------------------------------------------------------------- TMA tile load
// The p-pass tile is C columns (C = 1, 2, 4, 8) by NP rows of 16-byte elements,
// row-major, in the layout a 2-D tensor copy (cp.async.bulk.tensor) writes with
// the swizzle of a C * 16-byte row: none (C = 1), 32B (C = 2), 64B (C = 4) or
// 128B (C = 8), i.e. element (k, c) at k C + (c ^ tma_sw<C>(k)) -- the 16-byte
// chunk index XORed with address bits 7.. of the row.  Reading one column over
// consecutive rows then touches distinct 16-byte bank groups.
template <int C>
__host__ __device__ constexpr int tma_sw(int k) {
  return C == 1 ? 0 : ((k >> (C == 2 ? 2 : (C == 4 ? 1 : 0))) & (C - 1));
}
template <int C> struct TmaSlot {
  int c;
  __device__ __forceinline__ int operator()(int k) const { return k * C + (c ^ tma_sw<C>(k)); }
};

// A CUtensorMap as a kernel parameter (128 bytes, 64-byte aligned), encoded on the host.
struct __align__(64) TensorMap {
  unsigned long long v[16];
};

#ifdef WIG_TMA
__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

// Load rows [0, NP) of columns [col0, col0 + C) of the complex128 (NP, NX) array
// behind `map` into the tile at `tile` (1024-byte aligned) with 2-D tensor copies
// of BOXR rows each, completing on `bar`; every thread returns once the bytes have
// landed, or after a bounded wait (the status word then records WIG_ERR_TIMEOUT).
template <int NP, int C>
__device__ __forceinline__ void tma_tile_load(double2* tile, const TensorMap* map, int col0,
                                              unsigned long long* bar, int* status) {
  constexpr int BOXR = NP < 256 ? NP : 256;
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
                 "r"((unsigned)(C * NP * 16))
                 : "memory");
#pragma unroll 1
    for (int r = 0; r < NP; r += BOXR)
      asm volatile(
          "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
          "[%4];" ::"r"(smem_addr(tile + (size_t)r * C)),
          "l"(reinterpret_cast<unsigned long long>(map)), "r"(2 * col0), "r"(r), "r"(smem_addr(bar))
          : "memory");
  }
  __syncthreads();   // the barrier is initialised before anyone waits on it
  unsigned done = 0;
#pragma unroll 1
  for (long it = 0; it < (1L << 24) && !done; ++it)
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(smem_addr(bar))
        : "memory");
  if (!done && threadIdx.x == 0) atomicExch(status, 1);
}
#endif

// Column of a C-wide tile owned by group `grp` of warp `warp`; 8-lane groups
// pair columns c and c ^ PM so the two sequences of a half-warp use distinct
// bank pairs.
template <int N, int WARPS>
__device__ __forceinline__ int rf_tile_col(int warp, int grp) {
  constexpr int G = rf_g(N), SPW = rf_spw(N), C = WARPS * SPW;
  if constexpr (G == 8) {
    constexpr int PM = C / 2 < 8 ? C / 2 : 8;
    const int hw = 2 * warp + (grp >> 1);
    const int base = (hw & (PM - 1)) | ((hw / PM) * 2 * PM);
    return base ^ ((grp & 1) * PM);
  } else {
    return warp * SPW + grp;
  }
}

// x-pass: WARPS * rf_spw(NX) rows per CTA (xpass_body's arithmetic).
template <class Phys, int NX, int NP, int WARPS, bool KIN_STRING>
__device__ __forceinline__ void xpass_rf_body(const WigArgs& a, const Phys& ph, double2* __restrict__ W,
                                              int scale_mode, double* obs_row) {
  typedef RegFft<double2, NX> F;
  constexpr int E = F::E, G = F::G, Q = F::Q, SPW = rf_spw(NX), NT = WARPS * 32;
  constexpr int XS = NX + (G == 8 ? 8 : 0);
  extern __shared__ double2 sm[];
  __shared__ double red[NT / 32][NACC];
  double2 s = make_double2(1., 0.);
  if (scale_mode != 0 || (obs_row != nullptr && blockIdx.x == 0))
    s = consume_partials<NT>(a, scale_mode, blockIdx.x == 0 ? obs_row : nullptr, red);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, grp = lane / G, g = lane % G;
  const int seq = warp * SPW + grp;
  const int row = blockIdx.x * (WARPS * SPW) + seq;
  WIG_BOUNDS_CHECK("x-pass row", row, NP);
  double2* Wr = W + (size_t)row * NX;
  double2 v[E];
#pragma unroll
  for (int m = 0; m < E; ++m) {
    double2 u = Wr[g + G * m];
    if (scale_mode != 0) u = cmul(u, s);
    v[m] = u;
  }
  const SlotX<double2, PlainSlot> x{sm, PlainSlot{seq * XS}};
  F::fwdx(v, x, a.rtw_x, g);
  __syncwarp();
#pragma unroll
  for (int e = 0; e < E; ++e) x.put(g * Q + e / G + E * (e % G), v[e]);
  __syncwarp();
  const double inv_n = 1.0 / (double)NX;
  const int ii = (row + NP / 2) % NP;
  const double p = a.dp * (ii - 0.5 * NP);
#pragma unroll 1
  for (int k = g; k < NX; k += G) {
    const int jj = (k + NX / 2) % NX;
    const double lambda = a.dlambda * (jj - 0.5 * NX);
    double phase;
    if (KIN_STRING)
      phase = a.dt * ((ph.KineticEnergy(p + a.hbar * lambda / 2.) -
                       ph.KineticEnergy(p - a.hbar * lambda / 2.)) / a.hbar);
    else
      phase = a.dt * lambda * p / a.mass;
    const double rr = a.r_lambda[k] * inv_n;
    double sn, cs;
    sincos(phase, &sn, &cs);
    x.put(k, cmul(x.get(k), make_double2(rr * cs, -rr * sn)));
  }
  __syncwarp();
#pragma unroll
  for (int e = 0; e < E; ++e) v[e] = x.get(g * Q + e / G + E * (e % G));
  F::invx(v, x, a.rtw_x + NX, g);
#pragma unroll
  for (int m = 0; m < E; ++m) Wr[g + G * m] = v[m];
}

// p-pass of the Lie step: a tile of C = WARPS * rf_spw(NP) columns per CTA
// (ppass_body's arithmetic with HALF = 0, FINAL = 1, no Gross-Pitaevskii
// phase).  DAMP: 0 none, 1 Caldeira-Leggett; KVN: the classical factor.
// Shared memory: 1 KB of alignment slack, then A [NP][C] and (DAMP) B [NP][C] double2.
// With WIG_TMA the tile arrives by 2-D tensor copies (tma_tile_load, `map` over W),
// otherwise by coalesced thread loads into the same layout.
template <class Phys, int NX, int NP, int WARPS, int DAMP, int KVN>
__device__ __forceinline__ void ppass_rf_body(const WigArgs& a, const Phys& ph, double2* __restrict__ W, double t,
                                              double* __restrict__ partials, const TensorMap* map) {
  typedef RegFft<double2, NP> F;
  constexpr int E = F::E, G = F::G, Q = F::Q, SPW = rf_spw(NP), C = WARPS * SPW, NT = WARPS * 32;
  static_assert(C == 1 || C == 2 || C == 4 || C == 8, "tile of 1, 2, 4 or 8 columns");
  extern __shared__ double2 sm[];
  __shared__ double red[NT / 32][NACC];
  __shared__ __align__(8) unsigned long long tbar;
  double2* A = reinterpret_cast<double2*>((reinterpret_cast<unsigned long long>(sm) + 1023ull) & ~1023ull);
  double2* B = A + C * NP;
  const int col0 = blockIdx.x * C;
#ifdef WIG_TMA
  WIG_BOUNDS_CHECK("p-pass tile column", col0 + C - 1, NX);
  tma_tile_load<NP, C>(A, map, col0, &tbar, a.status);
#else
  for (int e = threadIdx.x; e < C * NP; e += NT) {
    const int k = e / C, c = e & (C - 1);
    WIG_BOUNDS_CHECK("p-pass tile column", col0 + c, NX);
    A[k * C + (c ^ tma_sw<C>(k))] = W[(size_t)k * NX + col0 + c];
  }
  __syncthreads();
  (void)map;
  (void)tbar;
#endif
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, grp = lane / G, g = lane % G;
  const int c = rf_tile_col<NP, WARPS>(warp, grp);
  const int col = col0 + c;
  const TmaSlot<C> sl{c};
  const SlotX<double2, TmaSlot<C>> xa{A, sl}, xb{B, sl};
  double2 w[E];
#pragma unroll
  for (int m = 0; m < E; ++m) w[m] = xa.get(g + G * m);
  F::fwdx(w, xa, a.rtw_p, g);
  __syncwarp();
#pragma unroll
  for (int e = 0; e < E; ++e) xa.put(g * Q + e / G + E * (e % G), w[e]);
  __syncwarp();
  const int jj = (col + NX / 2) % NX;
  const double x = a.dx * (jj - 0.5 * NX);
  const double m1 = a.mask1[col], m2 = a.mask2s[col];
#pragma unroll 1
  for (int k = g; k < NP; k += G) {
    const int ii = (k + NP / 2) % NP;
    const double theta = a.dtheta * (ii - 0.5 * NP);
    const double phase = KVN ? a.dt * (-ph.DPotential(t, x) * theta)
                             : a.dt * ((ph.Potential(t, x - a.hbar * theta / 2.) -
                                        ph.Potential(t, x + a.hbar * theta / 2.)) / a.hbar);
    const double r = a.r_theta[k];
    double sn, cs;
    sincos(phase, &sn, &cs);
    double2 v = cmul(xa.get(k), make_double2(r * cs, -r * sn));
    v = cscale(v, m1);
    v = cscale(v, m2);
    xa.put(k, v);
  }
  __syncwarp();
#pragma unroll
  for (int e = 0; e < E; ++e) w[e] = xa.get(g * Q + e / G + E * (e % G));
  F::invx(w, xa, a.rtw_p + NP, g);
  if (DAMP == 1) {
    // A + c3 D(A + c12 D(A + c1 D A)), D = IFFT_p[theta FFT_p(sign(p) f(p) .)] / n_p; A in the
    // column's A slots, the transforms exchanging through its B slots
    __syncwarp();
#pragma unroll
    for (int m = 0; m < E; ++m) xa.put(g + G * m, w[m]);
#pragma unroll 1
    for (int it = 0; it < 3; ++it) {
#pragma unroll
      for (int m = 0; m < E; ++m) w[m] = cscale(w[m], a.sfp[g + G * m]);
      F::fwdx(w, xb, a.rtw_p, g);
#pragma unroll
      for (int i = 0; i < Q; ++i)
#pragma unroll
        for (int b = 0; b < G; ++b) w[i * G + b] = cscale(w[i * G + b], a.theta_s[g * Q + i + E * b]);
      F::invx(w, xb, a.rtw_p + NP, g);
      const double2 cf = it == 0 ? a.cl_k1 : (it == 1 ? a.cl_k12 : a.cl_c3);
#pragma unroll
      for (int m = 0; m < E; ++m) w[m] = cadd(xa.get(g + G * m), cmul(cf, w[m]));
    }
  }
  double acc[NACC];
#pragma unroll
  for (int v = 0; v < NACC; ++v) acc[v] = 0.;
  const double xt = a.x_tab[col], dv = a.dV_tab[col], v0 = a.V0_tab[col];
#pragma unroll
  for (int m = 0; m < E; ++m) accumulate_obs(acc, w[m], xt, a.p_tab[g + G * m], dv, v0, a.mass_exact);
  __syncwarp();
#pragma unroll
  for (int m = 0; m < E; ++m) xa.put(g + G * m, w[m]);
  block_sum<NT, NACC>(acc, red);    // its barriers also order the tile writes before the store
  if (threadIdx.x < NACC) partials[(size_t)blockIdx.x * NACC + threadIdx.x] = red[0][threadIdx.x];
  for (int e = threadIdx.x; e < C * NP; e += NT) {
    const int k = e / C, c2 = e & (C - 1);
    W[(size_t)k * NX + col0 + c2] = A[k * C + (c2 ^ tma_sw<C>(k))];
  }
}

}  // namespace wig
