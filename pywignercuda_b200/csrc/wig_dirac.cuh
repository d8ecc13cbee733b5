// Dirac2D 4-spinor split-operator step for sm_100a: two fused passes per step.
//
// Layout: psi is (4, N_y, N_x) complex128, each component row-major, x
// contiguous, FFT-shifted (GPU_Dirac2D.py:331-332).
//
// The reference's step (GPU_Dirac2D.Run :1055-1105) is
//   observables(x) -> FFT2 -> Normalize_P -> <K> -> K mix -> IFFT2 -> A mix(t)
//   -> absorbing boundary -> Normalize_X.
// Split at the FFT2 / IFFT2 boundaries into
//   column pass: column FFT, p-space partial sums (norm, <K>, <px>, <py>),
//                K mix (BaseCUDAsource_K :74-117), column IFFT;
//   row pass:    row IFFT, A mix (DiracPropagatorA_source :123-222), absorbing
//                boundary (:225-283), x-space partial sums (<x>, <y>, <alpha>,
//                <beta>, <A0>, norm), row FFT of the next step.
// Normalize_P and Normalize_X are scalar multiplications: Normalize_P's factor
// (from the column pass's partials) is applied when the next row pass loads
// its rows, which also makes the preceding Normalize_X redundant for the
// propagated data (it is applied once, at the end of the run); the x-space
// observables are ratios of partial sums, so they come out normalised.
#pragma once
#include "wig_fft.cuh"
#include "wig_wigner.cuh"

namespace wig {

constexpr int DNR = 8;   // row-pass sums: rho, rho(before boundary), rho x, rho y, alpha1, alpha2, beta, A0 rho
constexpr int DNC = 6;   // col-pass sums: |q|^2, beta_p, px-mix, py-mix, |q|^2 px, |q|^2 py
constexpr int DNOBS = 10;

struct DiracArgs {
  // kernel constants as the reference's kernels see them (GPU_Dirac2D.py:358-367)
  double mass, c, dt, dX, dY, dPx, dPy;
  // exact host values
  double dX_e, dY_e, dPx_e, dPy_e, mass_e, c_e;
  const double* x_tab;   // [n_x] shifted X (exact)
  const double* y_tab;   // [n_y]
  const double* px_tab;  // [n_x] shifted Px (exact)
  const double* py_tab;  // [n_y]
  const double* bx;      // [2][n_x] absorbing factors along x
  const double* by;      // [2][n_y] absorbing factors along y
  const double2* tw_x;
  const double2* tw_y;
  double* part_row[2];   // [n_cta_row][DNR], ping-pong by row-pass parity
  double* part_col;      // [n_cta_col][DNC]
  int n_row_cta, n_col_cta;
  double coef[8];        // cf[0..7] of the expression strings
};

// ---------------------------------------------------------------- A mix
template <class Phys>
__device__ __forceinline__ void dirac_A(const DiracArgs& a, const Phys& ph, double t, double x, double y,
                                        double2& p1, double2& p2, double2& p3, double2& p4) {
  // The reference's pow(v, 2.) are squares and its repeated "* sF / F" one
  // ratio: written as products, the factors differ from it by rounding only.
  const double A0 = ph.A0(t, x, y), A1 = ph.A1(t, x, y), A2 = ph.A2(t, x, y), A3 = ph.A3(t, x, y);
  const double mc2 = a.mass * a.c * a.c;
  const double F = sqrt(mc2 * mc2 + a.c * (A1 * A1 + A2 * A2 + A3 * A3));
  double sv, cv;
  sincos(a.dt * A0, &sv, &cv);
  const double2 e = make_double2(cv, -sv);               // exp(-i dt A0)
  double sF, cF;
  sincos(a.dt * F, &sF, &cF);
  const double r = sF / F;
  const double2 U11 = make_double2(cF, -mc2 * r);
  const double2 U33 = make_double2(cF, mc2 * r);
  const double2 U31 = make_double2(0., A3 * r);
  const double2 U41 = make_double2(-A2 * r, A1 * r);
  const double2 U32 = make_double2(A2 * r, A1 * r);
  const double2 U42 = make_double2(0., -A3 * r);
  const double2 q1 = cmul(e, cadd(cadd(cmul(U11, p1), cmul(U31, p3)), cmul(U32, p4)));
  const double2 q2 = cmul(e, cadd(cadd(cmul(U11, p2), cmul(U41, p3)), cmul(U42, p4)));
  const double2 q3 = cmul(e, cadd(cadd(cmul(U31, p1), cmul(U32, p2)), cmul(U33, p3)));
  const double2 q4 = cmul(e, cadd(cadd(cmul(U41, p1), cmul(U42, p2)), cmul(U33, p4)));
  p1 = q1; p2 = q2; p3 = q3; p4 = q4;
}

__device__ __forceinline__ double n2(double2 v) { return v.x * v.x + v.y * v.y; }
// Re(a conj(b)), Im(a conj(b))
__device__ __forceinline__ double re_acb(double2 a, double2 b) { return a.x * b.x + a.y * b.y; }
__device__ __forceinline__ double im_acb(double2 a, double2 b) { return a.y * b.x - a.x * b.y; }

// Sample finalisation (one CTA): observables of a sample from the row sums of
// the row pass that produced the x-space state and the column sums of the
// column pass that followed (Average_X/Y/Alpha1/Alpha2/Beta, Potential_0_Average,
// Average_KEnergy; GPU_Dirac2D.py:808-934).
template <int NT>
__device__ __forceinline__ void dirac_finalize_sample(const DiracArgs& a, const double* prow, int nrow,
                                                      const double* pcol, int ncol, double* obs_row) {
  __shared__ double red[NT / 32][NACC];
  double acc[NACC];
#pragma unroll
  for (int v = 0; v < NACC; ++v) acc[v] = 0.;
  for (int i = threadIdx.x; i < nrow; i += NT) {
#pragma unroll
    for (int v = 0; v < DNR; ++v) acc[v] += prow[(size_t)i * DNR + v];
  }
  block_sum<NT, NACC>(acc, red);
  double R[DNR];
#pragma unroll
  for (int v = 0; v < DNR; ++v) R[v] = red[0][v];
  __syncthreads();
#pragma unroll
  for (int v = 0; v < NACC; ++v) acc[v] = 0.;
  for (int i = threadIdx.x; i < ncol; i += NT) {
#pragma unroll
    for (int v = 0; v < DNC; ++v) acc[v] += pcol[(size_t)i * DNC + v];
  }
  block_sum<NT, NACC>(acc, red);
  if (threadIdx.x == 0) {
    const double* Cp = red[0];
    const double S = R[0];
    obs_row[0] = R[2] / S;
    obs_row[1] = R[3] / S;
    obs_row[2] = 2. * R[4] / S;
    obs_row[3] = R[5] / S;
    obs_row[4] = R[6] / S;
    obs_row[5] = (a.mass_e * a.c_e * a.c_e * Cp[1] + a.c_e * (Cp[2] + Cp[3])) / Cp[0];
    obs_row[6] = R[7] / S;
    obs_row[7] = Cp[4] / Cp[0];
    obs_row[8] = Cp[5] / Cp[0];
    obs_row[9] = R[0] / R[1];   // the first row pass stores R[1] = R[0]
  }
  __syncthreads();
}

// Reduce column sums -> Normalize_P factor 1/sqrt(S dPx dPy) (Norm_P_GPU :948-957).
template <int NT>
__device__ __forceinline__ double dirac_p_scale(const DiracArgs& a, double (*red)[NACC]) {
  double acc[NACC];
#pragma unroll
  for (int v = 0; v < NACC; ++v) acc[v] = 0.;
  for (int i = threadIdx.x; i < a.n_col_cta; i += NT) acc[0] += a.part_col[(size_t)i * DNC];
  block_sum<NT, NACC>(acc, red);
  const double s = 1.0 / sqrt(red[0][0] * a.dPx_e * a.dPy_e);
  __syncthreads();
  return s;
}

// Row pass.  mode 0: first (load x-space psi, x sums, row FFT); 1: mid
// (row IFFT, A, boundary, x sums, row FFT); 2: last (row IFFT, A, boundary,
// x sums, store x-space).  parity selects the row-sum buffer written.
template <class Phys, int NX, int NY, int ROWS, int NT>
__device__ __forceinline__ void dirac_row_body(const DiracArgs& a, const Phys& ph, double2* __restrict__ psi,
                                               int mode, int parity, double t_step, double t_obs,
                                               double* obs_row) {
  typedef RowMap<NX> M;
  extern __shared__ double2 sm[];
  __shared__ double red[NT / 32][NACC];
  double scale = 1.0;
  if (mode != 0) scale = dirac_p_scale<NT>(a, red) * (1.0 / (double)NX);
  if (mode != 0 && blockIdx.x == 0 && obs_row != nullptr)
    dirac_finalize_sample<NT>(a, a.part_row[parity ^ 1], a.n_row_cta, a.part_col, a.n_col_cta, obs_row);
  const int row0 = blockIdx.x * ROWS;
  const size_t comp = (size_t)NX * NY;
  for (int e = threadIdx.x; e < 4 * ROWS * NX; e += NT) {
    const int b = e / NX, k = e - b * NX;          // b = m * ROWS + r
    const int m = b / ROWS, r = b - m * ROWS;
    double2 v = psi[m * comp + (size_t)(row0 + r) * NX + k];
    if (mode != 0) v = cscale(v, scale);
    sm[M::idx(b, k)] = v;
  }
  __syncthreads();
  if (mode != 0) cta_fft<double2, NX, 4 * ROWS, NT, true, M>(sm, a.tw_x);
  double acc[NACC];
#pragma unroll
  for (int v = 0; v < NACC; ++v) acc[v] = 0.;
  for (int e = threadIdx.x; e < ROWS * NX; e += NT) {
    const int r = e / NX, k = e - r * NX;
    const int row = row0 + r;
    const int id1 = M::idx(0 * ROWS + r, k), id2 = M::idx(1 * ROWS + r, k);
    const int id3 = M::idx(2 * ROWS + r, k), id4 = M::idx(3 * ROWS + r, k);
    double2 p1 = sm[id1], p2 = sm[id2], p3 = sm[id3], p4 = sm[id4];
    const int jj = (k + NX / 2) % NX, ii = (row + NY / 2) % NY;
    const double xk = a.dX * (double)(jj - NX / 2);
    const double yk = a.dY * (double)(ii - NY / 2);
    if (mode != 0) {
      dirac_A(a, ph, t_step, xk, yk, p1, p2, p3, p4);
      acc[1] += n2(p1) + n2(p2) + n2(p3) + n2(p4);
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const double bxq = a.bx[q * NX + k];
        p1 = cscale(p1, bxq); p2 = cscale(p2, bxq); p3 = cscale(p3, bxq); p4 = cscale(p4, bxq);
      }
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const double byq = a.by[q * NY + row];
        p1 = cscale(p1, byq); p2 = cscale(p2, byq); p3 = cscale(p3, byq); p4 = cscale(p4, byq);
      }
      sm[id1] = p1; sm[id2] = p2; sm[id3] = p3; sm[id4] = p4;
    }
    const double rho = n2(p1) + n2(p2) + n2(p3) + n2(p4);
    if (mode == 0) acc[1] += rho;
    acc[0] += rho;
    acc[2] += rho * a.x_tab[k];
    acc[3] += rho * a.y_tab[row];
    acc[4] += re_acb(p2, p3) + re_acb(p1, p4);
    acc[5] += -2. * (im_acb(p1, p4) + im_acb(p3, p2));
    acc[6] += n2(p1) + n2(p2) - n2(p3) - n2(p4);
    acc[7] += ph.A0(t_obs, xk, yk) * rho;
  }
  block_sum<NT, NACC>(acc, red);
  if (threadIdx.x < DNR) a.part_row[parity][(size_t)blockIdx.x * DNR + threadIdx.x] = red[0][threadIdx.x];
  if (mode != 2) cta_fft<double2, NX, 4 * ROWS, NT, false, M>(sm, a.tw_x);   // starts with the sync
  else __syncthreads();
  for (int e = threadIdx.x; e < 4 * ROWS * NX; e += NT) {
    const int b = e / NX, k = e - b * NX;
    const int m = b / ROWS, r = b - m * ROWS;
    psi[m * comp + (size_t)(row0 + r) * NX + k] = sm[M::idx(b, k)];
  }
}

// Column pass: tile of C columns x NY rows x 4 components; smem [k][m*C + c].
template <int NX, int NY, int C, int NT>
__device__ __forceinline__ void dirac_col_body(const DiracArgs& a, double2* __restrict__ psi) {
  typedef ColMap<4 * C> M;
  extern __shared__ double2 sm[];
  __shared__ double red[NT / 32][NACC];
  const int col0 = blockIdx.x * C;
  const size_t comp = (size_t)NX * NY;
  for (int e = threadIdx.x; e < 4 * C * NY; e += NT) {
    const int k = e / (4 * C), q = e - k * (4 * C);
    const int m = q / C, c = q - m * C;
    WIG_BOUNDS_CHECK("Dirac column-pass tile column", col0 + c, NX);
    sm[pad8(e)] = psi[m * comp + (size_t)k * NX + col0 + c];
  }
  __syncthreads();
  cta_fft<double2, NY, 4 * C, NT, false, M>(sm, a.tw_y);
  double acc[NACC];
#pragma unroll
  for (int v = 0; v < NACC; ++v) acc[v] = 0.;
  const double inv_ny = 1.0 / (double)NY;
  for (int e = threadIdx.x; e < C * NY; e += NT) {
    const int k = e / C, c = e - k * C;
    const int col = col0 + c;
    const int i1 = pad8(k * (4 * C) + c), i2 = pad8(k * (4 * C) + C + c);
    const int i3 = pad8(k * (4 * C) + 2 * C + c), i4 = pad8(k * (4 * C) + 3 * C + c);
    double2 q1 = sm[i1], q2 = sm[i2], q3 = sm[i3], q4 = sm[i4];
    const double pxe = a.px_tab[col], pye = a.py_tab[k];
    const double r2 = n2(q1) + n2(q2) + n2(q3) + n2(q4);
    acc[0] += r2;
    acc[1] += n2(q1) + n2(q2) - n2(q3) - n2(q4);
    acc[2] += pxe * (2. * (re_acb(q4, q1) + re_acb(q3, q2)));
    acc[3] += pye * (2. * (im_acb(q4, q1) + im_acb(q2, q3)));
    acc[4] += r2 * pxe;
    acc[5] += r2 * pye;
    // K mix (BaseCUDAsource_K :84-112), 1/NY of the column IFFT folded in
    const int jj = (col + NX / 2) % NX, ii = (k + NY / 2) % NY;
    const double px = a.dPx * (double)(jj - NX / 2);
    const double py = a.dPy * (double)(ii - NY / 2);
    const double pp = sqrt(px * px + py * py + pow(10., -12));
    double sn, cs;
    sincos(a.c * a.dt * pp, &sn, &cs);
    const double sdt = (sn / pp) * inv_ny;
    cs *= inv_ny;
    const double2 pplus = make_double2(py * sdt, px * sdt);    // (py + i px) sdt
    const double2 pminus = make_double2(py * sdt, -px * sdt);  // (py - i px) sdt
    sm[i1] = csub(cscale(q1, cs), cmul(pplus, q4));
    sm[i2] = cadd(cscale(q2, cs), cmul(pminus, q3));
    sm[i3] = cadd(cmul(make_double2(-pplus.x, -pplus.y), q2), cscale(q3, cs));
    sm[i4] = cadd(cmul(pminus, q1), cscale(q4, cs));
  }
  block_sum<NT, NACC>(acc, red);
  if (threadIdx.x < DNC) a.part_col[(size_t)blockIdx.x * DNC + threadIdx.x] = red[0][threadIdx.x];
  cta_fft<double2, NY, 4 * C, NT, true, M>(sm, a.tw_y);
  for (int e = threadIdx.x; e < 4 * C * NY; e += NT) {
    const int k = e / (4 * C), q = e - k * (4 * C);
    const int m = q / C, c = q - m * C;
    psi[m * comp + (size_t)k * NX + col0 + c] = sm[pad8(e)];
  }
}

// Final Normalize_X factor 1/sqrt(S dX dY) from the last row pass's sums.
template <int NT>
__device__ __forceinline__ void dirac_final_scale(const DiracArgs& a, int parity, double2* scale_out) {
  __shared__ double red[NT / 32][NACC];
  double acc[NACC];
#pragma unroll
  for (int v = 0; v < NACC; ++v) acc[v] = 0.;
  for (int i = threadIdx.x; i < a.n_row_cta; i += NT) acc[0] += a.part_row[parity][(size_t)i * DNR];
  block_sum<NT, NACC>(acc, red);
  if (threadIdx.x == 0) *scale_out = make_double2(1.0 / sqrt(red[0][0] * a.dX_e * a.dY_e), 0.);
}

}  // namespace wig
