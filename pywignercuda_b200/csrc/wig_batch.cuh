// Batched FP32 Wigner2D propagation: many independent instances of uneven
// grid sizes advanced together, one x-pass launch and one p-pass launch per
// step over a work list that spans every instance (x-items: blocks of rows,
// p-items: blocks of columns).  Each CTA's warps own whole sequences (rows or
// columns) and run the warp-level FP32 FFT of wig_fft32.cuh.
//
// Precision policy: W, FFTs and the pointwise factors are FP32 complex; FP64
// is used only to form the large phase arguments (dt*lambda*p/m and
// dt*[V(x - hbar theta/2) - V(x + hbar theta/2)]/hbar, the latter from the
// exact polynomial expansion) and to range-reduce them to [-pi, pi] before
// sincosf, and for the observables (FP64 Kahan-compensated sums per thread,
// FP64 tree / per-instance reductions).
//
// Normalisation (GPU_Wigner2D_FFT.Run :1912-1913): every p-item writes FP64
// partial sums; the last CTA of an instance to finish (arrival counter, no
// waiting) reduces them in item order, writes that step's observables and the
// instance's pending scale, which the next x-pass applies on load.
#pragma once
#include "wig_fft32.cuh"
#include "wig_wigner.cuh"

#ifndef WIGB_WARPS
#define WIGB_WARPS 8
#endif

namespace wig {

struct BInst {
  int n_x, n_p;
  int damp;          // 0 none, 1 Caldeira-Leggett
  int ff;            // f(p): 0 |p|, 1 p^2/sqrt(p^2 + f_eps)
  long long off;     // element offset in the packed state buffer
  int xitem0, n_xitems, pitem0, n_pitems;
  int tw_x, tw_p;    // offsets of the instance's twiddle tables in the table buffer
  double dt, hbar, mass, dx, dp, dtheta, dlambda, D_theta, D_lambda, f_eps;
  double v4, v2, v1, v0;   // V(x) = v4 x^4 + v2 x^2 + v1 x + v0
  double cl_k1, cl_k12, cl_c3;   // imaginary parts of the Caldeira-Leggett Horner coefficients
};

struct BArgs {
  const BInst* inst;
  const int2* xitems;    // (instance, first row)
  const int2* pitems;    // (instance, first column)
  float2* W;
  const float2* tw;
  double* partials;      // [n_pitems][NACC]
  unsigned* counters;    // [n_inst]
  double2* scale;        // [n_inst]
  double* obs;           // [n_inst][obs_stride][NOBS]
  int obs_stride;
};

// sequences per warp: enough that every stage of the warp FFT has >= 32
// butterflies (one or more per lane, no idle-lane branches)
__host__ __device__ constexpr int spw_of(int n) { return n >= 512 ? 1 : 512 / n; }

// Column stride of the p-pass tile (float2 units).  The transposing loads and
// stores put CPB consecutive columns of one row on consecutive lanes, a
// half-warp covering 16/CPB rows (8-byte accesses are served per half-warp):
// stride = 16/CPB (mod 16) spreads them over 16 distinct bank pairs; CPB >= 16
// needs an odd stride.
__host__ __device__ constexpr int col_stride(int n, int cpb) {
  return cpb >= 16 ? seq_stride32(n) + 1
                   : seq_stride32(n) + ((16 / cpb - seq_stride32(n) % 16) + 16) % 16;
}

// dt*lambda*p/m etc. reduced to [-pi, pi] in FP64 (two-term 2 pi, Cody-Waite)
__device__ __forceinline__ float reduce_phase(double phi) {
  const double q = rint(phi * 0.15915494309189533577);
  double r = fma(-q, 6.2831853071795862320, phi);
  r = fma(-q, 2.4492935982947063e-16, r);
  return (float)r;
}

struct Kahan {
  double s = 0., c = 0.;
  __device__ __forceinline__ void add(double v) {
    const double y = v - c, t = s + y;
    c = (t - s) - y;
    s = t;
  }
};

__device__ __forceinline__ void accumulate_obs_k(Kahan (&acc)[NACC], float2 v, double x, double p,
                                                 const BInst& I) {
  const double w = v.x;
  const double dV = (4. * I.v4 * x * x + 2. * I.v2) * x + I.v1;
  const double V = ((I.v4 * x * x + I.v2) * x + I.v1) * x + I.v0;
  acc[0].add(w);
  acc[1].add((double)v.y);
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

// Write this CTA's partials; the last CTA of the instance reduces them (item
// order, Kahan), writes the sample's observables and the instance's scale.
// mode: 0 none (scale 1), 1 normalise.
template <int NT>
__device__ __forceinline__ void batch_item_done(const BArgs& A, int inst, const BInst& I, int item,
                                                Kahan (&acc)[NACC], int mode, int sample) {
  __shared__ double red[NT / 32][NACC];
  __shared__ int s_last;
  double v[NACC];
#pragma unroll
  for (int k = 0; k < NACC; ++k) v[k] = acc[k].s + (-acc[k].c);
  block_sum<NT, NACC>(v, red);
  if (threadIdx.x < NACC) A.partials[(size_t)item * NACC + threadIdx.x] = red[0][threadIdx.x];
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = (atomicAdd(&A.counters[inst], 1u) == (unsigned)(I.n_pitems - 1));
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  __shared__ double tot[NACC];
  if (threadIdx.x < NACC) {
    Kahan k;
    for (int it = 0; it < I.n_pitems; ++it) k.add(__ldcg(&A.partials[(size_t)(I.pitem0 + it) * NACC + threadIdx.x]));
    tot[threadIdx.x] = k.s - k.c;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const double dXdP = I.dx * I.dp;
    const double2 S = make_double2(tot[0], tot[1]);
    double2 s = make_double2(1., 0.);
    if (mode == 1) s = crecip(make_double2(S.x * dXdP, S.y * dXdP));
    double* o = A.obs + ((size_t)inst * A.obs_stride + sample) * NOBS;
    o[0] = (s.x * S.x - s.y * S.y) * dXdP;
    for (int k = 1; k < NOBS; ++k) o[k] = s.x * (dXdP * tot[k + 1]);
    A.scale[inst] = s;
    A.counters[inst] = 0u;
  }
}

// ------------------------------------------------------------------ x-pass
template <int N>
__device__ __forceinline__ void batch_x_item(const BArgs& A, int inst, const BInst& I, int row0) {
  constexpr int SPW = spw_of(N);
  constexpr int SEQ = seq_stride32(N);
  extern __shared__ float2 smb[];
  float2* twsm = smb;                                   // [N]
  float* rtab = reinterpret_cast<float*>(smb + N);       // [N]
  float2* S = smb + N + (N + 1) / 2 + (threadIdx.x >> 5) * SPW * SEQ;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int m = threadIdx.x; m < N; m += blockDim.x) {
    if (m < stage_tw_size(N)) twsm[m] = A.tw[I.tw_x + m];
    const int jj = (m + N / 2) % N;
    const double lam = I.dlambda * (jj - 0.5 * N);
    rtab[m] = (float)(exp(-I.D_lambda * lam * lam) / (double)N);
  }
  const double2 sd = A.scale[inst];
  const float2 sc = make_float2((float)sd.x, (float)sd.y);
  float2* Wi = A.W + I.off;
  for (int sq = 0; sq < SPW; ++sq) {
    const int row = row0 + warp * SPW + sq;
    const float2* src = Wi + (size_t)row * N;
    for (int k = lane; k < N; k += 32) S[sq * SEQ + pad16(k)] = cmul(src[k], sc);
  }
  __syncthreads();
  warp_fft<N, SPW, false>(S, twsm, lane);
  for (int sq = 0; sq < SPW; ++sq) {
    const int row = row0 + warp * SPW + sq;
    const int ii = (row + I.n_p / 2) % I.n_p;
    const double p = I.dp * (ii - 0.5 * I.n_p);
    const double cp = I.dt * p / I.mass;
    for (int k = lane; k < N; k += 32) {
      const int jj = (k + N / 2) % N;
      const double lam = I.dlambda * (jj - 0.5 * N);
      float sn, cs;
      sincosf(reduce_phase(cp * lam), &sn, &cs);
      const float r = rtab[k];
      const int id = sq * SEQ + pad16(k);
      S[id] = cmul(S[id], make_float2(r * cs, -r * sn));
    }
  }
  __syncwarp();
  warp_fft<N, SPW, true>(S, twsm, lane);
  for (int sq = 0; sq < SPW; ++sq) {
    const int row = row0 + warp * SPW + sq;
    float2* dst = Wi + (size_t)row * N;
    for (int k = lane; k < N; k += 32) dst[k] = S[sq * SEQ + pad16(k)];
  }
}

// ------------------------------------------------------------------ p-pass
// Column tile of WIGB_WARPS*SPW columns, stored column-major in shared memory
// (column stride SEQ+1, odd, so the transposing loads/stores are conflict-free).
template <int N>
__device__ __forceinline__ void batch_cl_D(const BInst& I, float2* B, const float2* twsm, const float* sfp,
                                           const float* ths, int lane) {
  constexpr int SPW = spw_of(N);
  constexpr int CS = col_stride(N, WIGB_WARPS * SPW);
  for (int sq = 0; sq < SPW; ++sq)
    for (int k = lane; k < N; k += 32) B[sq * CS + pad16(k)] = cscale(B[sq * CS + pad16(k)], sfp[k]);
  __syncwarp();
  warp_fft_cs<N, SPW, CS, false>(B, twsm, lane);
  for (int sq = 0; sq < SPW; ++sq)
    for (int k = lane; k < N; k += 32) B[sq * CS + pad16(k)] = cscale(B[sq * CS + pad16(k)], ths[k]);
  __syncwarp();
  warp_fft_cs<N, SPW, CS, true>(B, twsm, lane);
}

template <int N>
__device__ __forceinline__ void batch_p_item(const BArgs& A, int inst, const BInst& I, int col0, int item,
                                             double t, int sample) {
  constexpr int SPW = spw_of(N);
  constexpr int CPB = WIGB_WARPS * SPW;
  constexpr int CS = col_stride(N, CPB);
  constexpr int NT = WIGB_WARPS * 32;
  extern __shared__ float2 smb[];
  float2* twsm = smb;                                     // [N] (per-stage twiddle tables)
  float* rth = reinterpret_cast<float*>(smb + N);          // [N] exp(-D theta^2 dt)
  float* sfp = rth + N;                                    // [N] sign(p) f(p)
  float* ths = sfp + N;                                    // [N] theta / N
  float2* tile = smb + N + (3 * N + 1) / 2;                // [CPB * CS]
  float2* btile = tile + CPB * CS;                         // [CPB * CS] (Caldeira-Leggett)
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nx = I.n_x;
  for (int m = threadIdx.x; m < N; m += NT) {
    if (m < stage_tw_size(N)) twsm[m] = A.tw[I.tw_p + m];
    const int ii = (m + N / 2) % N;
    const double th = I.dtheta * (ii - 0.5 * N);
    rth[m] = (float)exp(-I.D_theta * th * th * I.dt);
    const double p = I.dp * (ii - 0.5 * N);
    double f = (I.ff == 0) ? fabs(p) : p * p / sqrt(p * p + I.f_eps);
    sfp[m] = (float)(p >= 0. ? f : -f);
    ths[m] = (float)(th / (double)N);
  }
  float2* Wi = A.W + I.off;
  for (int e = threadIdx.x; e < CPB * N; e += NT) {
    const int k = e / CPB, c = e - k * CPB;
    tile[c * CS + pad16(k)] = Wi[(size_t)k * nx + col0 + c];
  }
  __syncthreads();
  float2* S = tile + warp * SPW * CS;
  warp_fft_cs<N, SPW, CS, false>(S, twsm, lane);
  const double xmax = I.dx * (nx - 1.) / 2.;
  for (int sq = 0; sq < SPW; ++sq) {
    const int col = col0 + warp * SPW + sq;
    const int jj = (col + nx / 2) % nx;
    const double x = I.dx * (jj - 0.5 * nx);
    const float m1 = (float)(1. - exp(-(x - xmax) * (x - xmax) / ((10. * I.dx) * (10. * I.dx))));
    const float m2 = (float)((1. - exp(-(x + xmax) * (x + xmax) / ((10. * I.dx) * (10. * I.dx)))) / (double)N);
    const float mm = m1 * m2;
    // V(x - u) - V(x + u) = -2u (4 v4 x^3 + 4 v4 x u^2 + 2 v2 x + v1), u = hbar theta / 2
    const double a3 = 4. * I.v4 * x * x * x + 2. * I.v2 * x + I.v1, a1 = 4. * I.v4 * x;
    const double ph0 = -I.dt / I.hbar;
    for (int k = lane; k < N; k += 32) {
      const int ii = (k + N / 2) % N;
      const double th = I.dtheta * (ii - 0.5 * N);
      const double u = 0.5 * I.hbar * th;
      const double dV = -2. * u * (a3 + a1 * u * u);
      float sn, cs;
      sincosf(reduce_phase(-ph0 * dV), &sn, &cs);
      const float r = rth[k] * mm;
      const int id = sq * CS + pad16(k);
      S[id] = cmul(S[id], make_float2(r * cs, -r * sn));
    }
  }
  __syncwarp();
  warp_fft_cs<N, SPW, CS, true>(S, twsm, lane);
  if (I.damp == 1) {
    float2* Bw = btile + warp * SPW * CS;
    const float2 k1 = make_float2(0.f, (float)I.cl_k1), k12 = make_float2(0.f, (float)I.cl_k12);
    const float2 c3 = make_float2(0.f, (float)I.cl_c3);
    for (int sq = 0; sq < SPW; ++sq)
      for (int k = lane; k < N; k += 32) Bw[sq * CS + pad16(k)] = S[sq * CS + pad16(k)];
    __syncwarp();
    batch_cl_D<N>(I, Bw, twsm, sfp, ths, lane);
    for (int sq = 0; sq < SPW; ++sq)
      for (int k = lane; k < N; k += 32) {
        const int id = sq * CS + pad16(k);
        Bw[id] = cadd(S[id], cmul(k1, Bw[id]));
      }
    __syncwarp();
    batch_cl_D<N>(I, Bw, twsm, sfp, ths, lane);
    for (int sq = 0; sq < SPW; ++sq)
      for (int k = lane; k < N; k += 32) {
        const int id = sq * CS + pad16(k);
        Bw[id] = cadd(S[id], cmul(k12, Bw[id]));
      }
    __syncwarp();
    batch_cl_D<N>(I, Bw, twsm, sfp, ths, lane);
    for (int sq = 0; sq < SPW; ++sq)
      for (int k = lane; k < N; k += 32) {
        const int id = sq * CS + pad16(k);
        S[id] = cadd(S[id], cmul(c3, Bw[id]));
      }
  }
  __syncthreads();
  Kahan acc[NACC];
  for (int e = threadIdx.x; e < CPB * N; e += NT) {
    const int k = e / CPB, c = e - k * CPB;
    const int col = col0 + c;
    const float2 v = tile[c * CS + pad16(k)];
    Wi[(size_t)k * nx + col] = v;
    const int jj = (col + nx / 2) % nx, ii = (k + N / 2) % N;
    accumulate_obs_k(acc, v, I.dx * (jj - 0.5 * nx), I.dp * (ii - 0.5 * N), I);
  }
  batch_item_done<NT>(A, inst, I, item, acc, I.damp ? 1 : 0, sample);
  (void)t;
}

// Initial normalisation and sample 0 (Run :1778-1780), over the p-items.
template <int N>
__device__ __forceinline__ void batch_reduce_item(const BArgs& A, int inst, const BInst& I, int col0, int item,
                                                  int mode, int sample) {
  constexpr int SPW = spw_of(N);
  constexpr int CPB = WIGB_WARPS * SPW;
  constexpr int NT = WIGB_WARPS * 32;
  const int nx = I.n_x;
  const float2* Wi = A.W + I.off;
  Kahan acc[NACC];
  for (int e = threadIdx.x; e < CPB * N; e += NT) {
    const int k = e / CPB, c = e - k * CPB;
    const int col = col0 + c;
    const int jj = (col + nx / 2) % nx, ii = (k + N / 2) % N;
    accumulate_obs_k(acc, Wi[(size_t)k * nx + col], I.dx * (jj - 0.5 * nx), I.dp * (ii - 0.5 * N), I);
  }
  batch_item_done<NT>(A, inst, I, item, acc, mode, sample);
}

template <int N>
__device__ __forceinline__ void batch_scale_item(const BArgs& A, int inst, const BInst& I, int col0) {
  constexpr int SPW = spw_of(N);
  constexpr int CPB = WIGB_WARPS * SPW;
  constexpr int NT = WIGB_WARPS * 32;
  const double2 sd = A.scale[inst];
  const float2 sc = make_float2((float)sd.x, (float)sd.y);
  float2* Wi = A.W + I.off;
  for (int e = threadIdx.x; e < CPB * N; e += NT) {
    const int k = e / CPB, c = e - k * CPB;
    const size_t g = (size_t)k * I.n_x + col0 + c;
    Wi[g] = cmul(Wi[g], sc);
  }
}

}  // namespace wig
