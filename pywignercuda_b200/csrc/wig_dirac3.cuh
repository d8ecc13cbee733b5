// Dirac3D 4-spinor split-operator step for sm_100a: four fused passes per step.
//
// Layout: psi is (4, N_z, N_y, N_x) complex128, each component (z, y, x)
// row-major with x contiguous, every axis FFT-shifted (GPU_Dirac3D.py:659-661).
//
// The reference's step (GPU_Dirac3D.Run :1325-1465) is
//   position averages(t) -> FFT3 -> [momentum averages] -> K mix -> IFFT3 / N
//   -> A mix(t)
// with one normalisation before the loop.  Cut at the axis transforms:
//   x-pass:  row IFFT (x), A mix of the previous step, position partial sums of
//            the next sample, row FFT (x)                     [one row = x line]
//   y-pass:  column FFT (y)                                    [per component]
//   z-pass:  column FFT (z), momentum partial sums, K mix (with the 1/N of the
//            IFFT3), column IFFT (z)                           [4 components]
//   y-pass:  column IFFT (y)
// so a step reads and writes the spinor four times (512 B per grid point).  The
// first x-pass of a run has no IFFT / A; the last has no sums / FFT and leaves
// the spinor in position space.  Every pass is grid-stride over its tiles, so
// each CTA writes one row of partial sums; the x-pass's block 0 turns the sums
// of the previous sample into its observables (fixed order, deterministic).
#pragma once
#include "wig_fft.cuh"
#include "wig_wigner.cuh"

namespace wig {

constexpr int D3X = 8;     // x-pass sums: rho, rho x, rho y, rho z, alpha1, alpha2, alpha3, A0 rho
constexpr int D3P = 5;     // z-pass sums: |q|^2, |q|^2 px, |q|^2 py, |q|^2 pz, K weight
constexpr int D3NOBS = 12;

struct Dirac3Args {
  // kernel constants as the reference's kernels see them (GPU_Dirac3D.py:690-700)
  double hbar, mass, c, dt, dX, dY, dZ, dPx, dPy, dPz;
  // exact host values (the Python-side products in Run and Norm_GPU)
  double dX_e, dY_e, dZ_e, dPx_e, dPy_e, dPz_e;
  const double2* tw_x;
  const double2* tw_y;
  const double2* tw_z;
  double* part_x[2];     // [n_x_cta][D3X], ping-pong by x-pass parity
  double* part_p;        // [n_z_cta][D3P]
  double* s1;            // [1] momentum-space sum of the step-1 spectrum (0: not yet known)
  double* scale;         // [1] factor of the initial Normalize_GPU
  int n_x_cta, n_z_cta;
  double coef[8];
};

__device__ __forceinline__ double d3_n2(double2 v) { return v.x * v.x + v.y * v.y; }
// Re(a conj(b)), Im(a conj(b))
__device__ __forceinline__ double d3_re(double2 a, double2 b) { return a.x * b.x + a.y * b.y; }
__device__ __forceinline__ double d3_im(double2 a, double2 b) { return a.y * b.x - a.x * b.y; }

// kernel coordinate delta (j - N/2), j = (idx + N/2) % N (every Dirac3D kernel)
__device__ __forceinline__ double d3_coord(double delta, int idx, int n) {
  return delta * (double)(((idx + n / 2) % n) - n / 2);
}

// ---------------------------------------------------------------- A mix
// DiracPropagatorA_source (:455-559): exp(-i dt A0) U(F), half the mass.
template <class Phys>
__device__ __forceinline__ void d3_A(const Dirac3Args& a, const Phys& ph, double t, double x, double y, double z,
                                     double2& p1, double2& p2, double2& p3, double2& p4) {
  const double A0 = ph.A0(t, x, y, z), A1 = ph.A1(t, x, y, z), A2 = ph.A2(t, x, y, z), A3 = ph.A3(t, x, y, z);
  const double m_ = 0.5 * a.mass;
  const double F = sqrt(pow(m_ * a.c * a.c, 2.) + (pow(A1, 2.) + pow(A2, 2.) + pow(A3, 2.)));
  const double om = F / a.hbar;
  double sv, cv;
  sincos(-a.dt * A0, &sv, &cv);
  const double2 e = make_double2(cv, sv);                 // exp(-i dt A0)
  double sF, cF;
  sincos(a.dt * om, &sF, &cF);
  const double sf = sF / F;
  const double2 U11 = make_double2(cF, -m_ * a.c * a.c * sf);
  const double2 U33 = make_double2(cF, m_ * a.c * a.c * sf);
  const double2 U13 = make_double2(0., A3 * sf);          // = U31
  const double2 U14 = make_double2(A2 * sf, A1 * sf);     // i A_-  = U32
  const double2 U23 = make_double2(-A2 * sf, A1 * sf);    // i A_+  = U41
  const double2 U24 = make_double2(0., -A3 * sf);         // = U42
  const double2 q1 = cmul(e, cadd(cadd(cmul(U11, p1), cmul(U13, p3)), cmul(U14, p4)));
  const double2 q2 = cmul(e, cadd(cadd(cmul(U11, p2), cmul(U23, p3)), cmul(U24, p4)));
  const double2 q3 = cmul(e, cadd(cadd(cmul(U13, p1), cmul(U14, p2)), cmul(U33, p3)));
  const double2 q4 = cmul(e, cadd(cadd(cmul(U23, p1), cmul(U24, p2)), cmul(U33, p4)));
  p1 = q1; p2 = q2; p3 = q3; p4 = q4;
}

// ---------------------------------------------------------------- sample finalisation
// Observables of one sample (one CTA) from the x-pass sums that preceded its
// FFT3 and the z-pass sums of its spectrum: Average_X/Y/Z (:1342-1352 -- sum
// times dX dY dZ), Average_Alpha1/2/3 (:1221-1249), Potential_0_Average
// (:1358-1361), Average_Px/Py/Pz and K_Energy_Average on the spectrum divided by
// the step-1 momentum norm (:1366-1395).  sample_tindex is the reference's
// t_index of the sample: at 1 the momentum norm is taken (Norm_P_GPU) and kept.
template <int NT>
__device__ __forceinline__ void d3_finalize_sample(const Dirac3Args& a, const double* px_part, long long sample_tindex,
                                                   double* obs_row) {
  __shared__ double red[NT / 32][NACC];
  double acc[NACC];
#pragma unroll
  for (int v = 0; v < NACC; ++v) acc[v] = 0.;
  for (int i = threadIdx.x; i < a.n_x_cta; i += NT) {
#pragma unroll
    for (int v = 0; v < D3X; ++v) acc[v] += px_part[(size_t)i * D3X + v];
  }
  block_sum<NT, NACC>(acc, red);
  double R[D3X];
#pragma unroll
  for (int v = 0; v < D3X; ++v) R[v] = red[0][v];
  __syncthreads();
#pragma unroll
  for (int v = 0; v < NACC; ++v) acc[v] = 0.;
  for (int i = threadIdx.x; i < a.n_z_cta; i += NT) {
#pragma unroll
    for (int v = 0; v < D3P; ++v) acc[v] += a.part_p[(size_t)i * D3P + v];
  }
  block_sum<NT, NACC>(acc, red);
  if (threadIdx.x == 0) {
    const double* Pp = red[0];
    double s1 = *a.s1;
    if (sample_tindex == 1 || !(s1 > 0.)) { s1 = Pp[0]; *a.s1 = s1; }
    const double dV = a.dX_e * a.dY_e * a.dZ_e;
    obs_row[0] = R[1] * a.dX_e * a.dY_e * a.dZ_e;
    obs_row[1] = R[2] * a.dX_e * a.dY_e * a.dZ_e;
    obs_row[2] = R[3] * a.dX_e * a.dY_e * a.dZ_e;
    obs_row[3] = R[4] * dV;
    obs_row[4] = R[5] * dV;
    obs_row[5] = R[6] * dV;
    obs_row[6] = R[7] * a.dX_e * a.dY_e * a.dZ_e;
    // |psi / norm|^2 dP = |psi|^2 / S1 with norm^2 = S1 dPx dPy dPz
    obs_row[7] = Pp[1] / s1;
    obs_row[8] = Pp[2] / s1;
    obs_row[9] = Pp[3] / s1;
    obs_row[10] = Pp[4] / s1;
    obs_row[11] = R[0] * dV;
  }
  __syncthreads();
}

// ---------------------------------------------------------------- x-pass
// mode 0: first of a run (load, scale by *a.scale when `normalise`, sums, row FFT);
// mode 1: row IFFT, A(t_A), sums at t_obs, row FFT; mode 2: row IFFT, A(t_A), store.
// Modes 1 and 2 finalise the previous sample (partials of parity ^ 1) into obs_prev.
template <class Phys, int NX, int NY, int NZ, int ROWS, int NT, int MAXR = 8>
__device__ __forceinline__ void d3_xpass_body(const Dirac3Args& a, const Phys& ph, double2* __restrict__ psi,
                                              int mode, int parity, int normalise, double t_A, double t_obs,
                                              long long prev_tindex, double* obs_prev) {
  typedef RowMap<NX> M;
  extern __shared__ double2 sm[];
  __shared__ double red[NT / 32][NACC];
  if (mode != 0 && blockIdx.x == 0 && obs_prev != nullptr)
    d3_finalize_sample<NT>(a, a.part_x[parity ^ 1], prev_tindex, obs_prev);
  const double scale = (mode == 0 && normalise) ? *a.scale : 1.0;
  constexpr int NROW = NY * NZ, NG = NROW / ROWS;
  const size_t comp = (size_t)NX * NROW;
  double acc[NACC];
#pragma unroll
  for (int v = 0; v < NACC; ++v) acc[v] = 0.;
  for (int g = blockIdx.x; g < NG; g += gridDim.x) {
    const int row0 = g * ROWS;
    for (int e = threadIdx.x; e < 4 * ROWS * NX; e += NT) {
      const int b = e / NX, k = e - b * NX;          // b = m * ROWS + r
      const int m = b / ROWS, r = b - m * ROWS;
      double2 v = psi[m * comp + (size_t)(row0 + r) * NX + k];
      if (mode == 0 && normalise) v = cscale(v, scale);
      sm[M::idx(b, k)] = v;
    }
    __syncthreads();
    if (mode != 0) {
      cta_fft<double2, NX, 4 * ROWS, NT, true, M, MAXR>(sm, a.tw_x);
      __syncthreads();   // explicit barrier before the pointwise mix, as in the z-pass
    }
    for (int e = threadIdx.x; e < ROWS * NX; e += NT) {
      const int r = e / NX, k = e - r * NX;
      const int row = row0 + r, iz = row / NY, iy = row - iz * NY;
      const int id1 = M::idx(0 * ROWS + r, k), id2 = M::idx(1 * ROWS + r, k);
      const int id3 = M::idx(2 * ROWS + r, k), id4 = M::idx(3 * ROWS + r, k);
      double2 p1 = sm[id1], p2 = sm[id2], p3 = sm[id3], p4 = sm[id4];
      const double x = d3_coord(a.dX, k, NX), y = d3_coord(a.dY, iy, NY), z = d3_coord(a.dZ, iz, NZ);
      if (mode != 0) {
        d3_A(a, ph, t_A, x, y, z, p1, p2, p3, p4);
        sm[id1] = p1; sm[id2] = p2; sm[id3] = p3; sm[id4] = p4;
      }
      if (mode != 2) {
        const double rho = d3_n2(p1) + d3_n2(p2) + d3_n2(p3) + d3_n2(p4);
        acc[0] += rho;
        acc[1] += rho * x;
        acc[2] += rho * y;
        acc[3] += rho * z;
        // Re of the dot sums of Average_Alpha1/2/3 (pycuda dot: no conjugation of the first)
        acc[4] += 2. * (d3_re(p4, p1) + d3_re(p3, p2));
        acc[5] += -2. * (d3_im(p1, p4) + d3_im(p3, p2));
        acc[6] += 2. * (d3_re(p3, p1) - d3_re(p4, p2));
        acc[7] += ph.A0(t_obs, x, y, z) * rho;
      }
    }
    __syncthreads();   // cta_fft's first stage reads shared memory before its first barrier
    if (mode != 2) cta_fft<double2, NX, 4 * ROWS, NT, false, M, MAXR>(sm, a.tw_x);
    for (int e = threadIdx.x; e < 4 * ROWS * NX; e += NT) {
      const int b = e / NX, k = e - b * NX;
      const int m = b / ROWS, r = b - m * ROWS;
      psi[m * comp + (size_t)(row0 + r) * NX + k] = sm[M::idx(b, k)];
    }
    __syncthreads();
  }
  if (mode != 2) {
    block_sum<NT, NACC>(acc, red);
    if (threadIdx.x < D3X) a.part_x[parity][(size_t)blockIdx.x * D3X + threadIdx.x] = red[0][threadIdx.x];
  }
}

// ---------------------------------------------------------------- y-pass
// One tile = component m, plane z, columns x0 .. x0 + C - 1, all NY rows.
template <int NX, int NY, int NZ, int C, int NT, bool INV, int MAXR = 8>
__device__ __forceinline__ void d3_ypass_body(const Dirac3Args& a, double2* __restrict__ psi) {
  typedef ColMap<C> M;
  extern __shared__ double2 sm[];
  constexpr int NCT = NX / C, NTILE = 4 * NZ * NCT;
  for (int g = blockIdx.x; g < NTILE; g += gridDim.x) {
    const int plane = g / NCT, x0 = (g - plane * NCT) * C;          // plane = m * NZ + z
    double2* base = psi + (size_t)plane * NX * NY + x0;
    for (int e = threadIdx.x; e < NY * C; e += NT) {
      const int k = e / C, c = e - k * C;
      sm[pad8(e)] = base[(size_t)k * NX + c];
    }
    __syncthreads();
    cta_fft<double2, NY, C, NT, INV, M, MAXR>(sm, a.tw_y);
    for (int e = threadIdx.x; e < NY * C; e += NT) {
      const int k = e / C, c = e - k * C;
      base[(size_t)k * NX + c] = sm[pad8(e)];
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------- z-pass
// One tile = row y, columns x0 .. x0 + C - 1, all NZ planes, 4 components;
// smem [z][m C + c].  K mix: DiracPropagatorK_source (:386-452), half the mass.
template <int NX, int NY, int NZ, int C, int NT, int MAXR = 8>
__device__ __forceinline__ void d3_zpass_body(const Dirac3Args& a, double2* __restrict__ psi) {
  typedef ColMap<4 * C> M;
  extern __shared__ double2 sm[];
  __shared__ double red[NT / 32][NACC];
  constexpr int NCT = NX / C, NTILE = NY * NCT;
  const size_t comp = (size_t)NX * NY * NZ, plane = (size_t)NX * NY;
  const double inv_n = 1.0 / ((double)NX * (double)NY * (double)NZ);
  const double m_ = 0.5 * a.mass;
  double acc[NACC];
#pragma unroll
  for (int v = 0; v < NACC; ++v) acc[v] = 0.;
  for (int g = blockIdx.x; g < NTILE; g += gridDim.x) {
    const int iy = g / NCT, x0 = (g - iy * NCT) * C;
    for (int e = threadIdx.x; e < 4 * C * NZ; e += NT) {
      const int k = e / (4 * C), q = e - k * (4 * C);
      const int m = q / C, c = q - m * C;
      sm[pad8(e)] = psi[m * comp + (size_t)k * plane + (size_t)iy * NX + x0 + c];
    }
    __syncthreads();
    cta_fft<double2, NZ, 4 * C, NT, false, M, MAXR>(sm, a.tw_z);
    // cta_fft ends with a barrier, yet on B200 the K mix below read stale spectra
    // (scattered tiles, about half the points at 16^3 and 32^3) unless this explicit
    // barrier follows the transform; with it the pass matches numpy to 3e-16
    __syncthreads();
    const double py = d3_coord(a.dPy, iy, NY);
    for (int e = threadIdx.x; e < C * NZ; e += NT) {
      const int k = e / C, c = e - k * C;
      const int i1 = pad8(k * (4 * C) + c), i2 = pad8(k * (4 * C) + C + c);
      const int i3 = pad8(k * (4 * C) + 2 * C + c), i4 = pad8(k * (4 * C) + 3 * C + c);
      const double2 q1 = sm[i1], q2 = sm[i2], q3 = sm[i3], q4 = sm[i4];
      const double px = d3_coord(a.dPx, x0 + c, NX), pz = d3_coord(a.dPz, k, NZ);
      const double r2 = d3_n2(q1) + d3_n2(q2) + d3_n2(q3) + d3_n2(q4);
      acc[0] += r2;
      acc[1] += r2 * px;
      acc[2] += r2 * py;
      acc[3] += r2 * pz;
      // K_Energy_Average_source (:27-89): full mass
      acc[4] += a.mass * a.c * a.c * (d3_n2(q1) + d3_n2(q2) - d3_n2(q3) - d3_n2(q4)) +
                2. * a.c * px * (d3_re(q4, q1) + d3_re(q3, q2)) +
                2. * a.c * py * (d3_im(q4, q1) + d3_im(q2, q3)) +
                2. * a.c * pz * (d3_re(q3, q1) - d3_re(q4, q2));
      // K mix, with the 1/(NX NY NZ) of the inverse transform folded in
      const double E = a.c * sqrt(px * px + py * py + pz * pz + pow(m_ * a.c, 2));
      double sn, cs;
      sincos(E * a.dt / a.hbar, &sn, &cs);
      const double sE = a.c * sn / E;
      const double2 U11 = make_double2(cs, -a.c * m_ * sE);
      const double2 U33 = make_double2(cs, a.c * m_ * sE);
      const double2 U13 = make_double2(0., -pz * sE);       // = U31
      const double2 U14 = make_double2(-py * sE, -px * sE);  // -(py + i px) c s / E   = U32
      const double2 U23 = make_double2(py * sE, -px * sE);   //  (py - i px) c s / E   = U41
      const double2 U24 = make_double2(0., pz * sE);        // = U42
      sm[i1] = cscale(cadd(cadd(cmul(U11, q1), cmul(U13, q3)), cmul(U14, q4)), inv_n);
      sm[i2] = cscale(cadd(cadd(cmul(U11, q2), cmul(U23, q3)), cmul(U24, q4)), inv_n);
      sm[i3] = cscale(cadd(cadd(cmul(U13, q1), cmul(U14, q2)), cmul(U33, q3)), inv_n);
      sm[i4] = cscale(cadd(cadd(cmul(U23, q1), cmul(U24, q2)), cmul(U33, q4)), inv_n);
    }
    __syncthreads();   // cta_fft's first stage reads shared memory before its first barrier
    cta_fft<double2, NZ, 4 * C, NT, true, M, MAXR>(sm, a.tw_z);
    for (int e = threadIdx.x; e < 4 * C * NZ; e += NT) {
      const int k = e / (4 * C), q = e - k * (4 * C);
      const int m = q / C, c = q - m * C;
      psi[m * comp + (size_t)k * plane + (size_t)iy * NX + x0 + c] = sm[pad8(e)];
    }
    __syncthreads();
  }
  block_sum<NT, NACC>(acc, red);
  if (threadIdx.x < D3P) a.part_p[(size_t)blockIdx.x * D3P + threadIdx.x] = red[0][threadIdx.x];
}

// ---------------------------------------------------------------- normalisation
// Normalize_GPU (:1144-1161): per-CTA sums of |psi|^2, then 1/sqrt(S dX dY dZ).
template <int NT>
__device__ __forceinline__ void d3_norm_body(const Dirac3Args& a, const double2* __restrict__ psi, long n) {
  __shared__ double red[NT / 32][NACC];
  double acc[NACC];
#pragma unroll
  for (int v = 0; v < NACC; ++v) acc[v] = 0.;
  for (long i = (long)blockIdx.x * NT + threadIdx.x; i < n; i += (long)gridDim.x * NT) acc[0] += d3_n2(psi[i]);
  block_sum<NT, NACC>(acc, red);
  if (threadIdx.x == 0) a.part_x[1][blockIdx.x] = red[0][0];
}

template <int NT>
__device__ __forceinline__ void d3_norm_final(const Dirac3Args& a, int n_cta) {
  __shared__ double red[NT / 32][NACC];
  double acc[NACC];
#pragma unroll
  for (int v = 0; v < NACC; ++v) acc[v] = 0.;
  for (int i = threadIdx.x; i < n_cta; i += NT) acc[0] += a.part_x[1][i];
  block_sum<NT, NACC>(acc, red);
  if (threadIdx.x == 0) {
    *a.scale = 1.0 / sqrt(red[0][0] * a.dX_e * a.dY_e * a.dZ_e);
    *a.s1 = 0.;
  }
}

}  // namespace wig
