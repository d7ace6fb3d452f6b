// Fast diagonalization of a doubly periodic system by Bloch waves.
//
// On a periodic direction of nel equal elements of order p the assembled 1-D
// stiffness K and weights W are block-circulant (p x p blocks, one per
// element, coupling only neighbouring elements). A Bloch wave
// x(e, i) = exp(i th_m e) v_i, th_m = 2 pi m / nel, reduces K v = mu W v to
// nel independent p x p Hermitian problems
//   K_m[i][j] = Kh[i][j] + [i=j=0] Kh[p][p] + [j=0] Kh[i][p] e^{i th}
//             + [i=0] Kh[p][j] e^{-i th},   W_m = diag(w_i + [i=0] w_p),
// so the 1-D eigenvectors are E[(e,i)][(m,k)] = e^{i th_m e} V_m[i][k]: a
// DFT across elements followed by a p x p multiply per wavenumber. The 2-D
// inverse A^{-1} = (E_y (x) E_x) D^{-1} (E_y (x) E_x)^H then costs three
// passes over the 512 x 512 array instead of four dense 512^3 products:
//   bloch_x_forward   one row y per block: radix-2 FFT over the
//                     elements for each local index, then V_m^H, for the
//                     wavenumbers m = 0..nel/2 (the input is real);
//   bloch_y_solve     one x mode (m_x, k_x) per block: FFT over the y
//                     elements, V^H, the spectral divide by
//                     alpha + bx mu_x + by mu_y (null modes to 0), V, inverse
//                     FFT;
//   bloch_x_backward  one row per block: V_m, the other half of the
//                     wavenumbers by conjugate symmetry (the result is real),
//                     inverse FFT, store or accumulate.
// The passes are latency-bound: one row (mode) per block, at most 32
// registers a thread (8 blocks per SM) and the twiddles in shared memory,
// so that a whole pass fits one wave.
// The spectral array is complex, column-major over the x modes
// ([(m_x, k_x)][y]). Element counts are powers of two (the FFT); the
// twiddles are tabulated on the host in extended precision. The FFT's
// rounding grows like log2(nel), where a dense transform's grows with the
// square root of its length: with eigenvectors accurate to the FP64
// rounding, one refinement step reaches about 6e-11 of the right-hand side
// at the bench's 64 x 64 elements of order 8.
#include "common.cuh"

namespace seg {
namespace {

constexpr int kBlochThreads = 256;
constexpr int kBlochMaxP = SE_MAXN;  // the sums over a block's p terms unroll to this

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
// conj(a) b
__device__ __forceinline__ double2 cmulc(double2 a, double2 b) {
  return make_double2(fma(a.x, b.x, a.y * b.y), fma(a.x, b.y, -a.y * b.x));
}
__device__ __forceinline__ int bitrev(int v, int logn) {
  return logn == 0 ? 0 : (int)(__brev((unsigned)v) >> (32 - logn));
}

// In-place radix-2 FFTs of length n = 2^logn on nseq sequences S[s][0..n)
// (stride n), input in bit-reversed order, output in natural order.
// inverse: conjugate twiddles. Unnormalised.
__device__ void fft_seqs(double2* S, int nseq, int n, int logn, const double2* tw, bool inverse) {
  const int nb = nseq * (n / 2);
  for (int s = 1; s <= logn; s++) {
    const int m2 = 1 << s, half = m2 >> 1, step = n / m2;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) {
      const int q = b / (n / 2), j = b - q * (n / 2);
      const int grp = j / half, pos = j - grp * half;
      double2* x = S + q * n;
      const int k0 = grp * m2 + pos, k1 = k0 + half;
      double2 w = tw[pos * step];
      if (inverse) w.y = -w.y;
      const double2 u = x[k0], v = cmul(x[k1], w);
      x[k0] = make_double2(u.x + v.x, u.y + v.y);
      x[k1] = make_double2(u.x - v.x, u.y - v.y);
    }
    __syncthreads();
  }
}

// R consecutive rows y0..y0+R-1 of the real G_y x G_x array F (rows past
// G_y skipped): S[r][i][m] = sum_e F(e, i) e^{-i th_m e}, then
// xh[(m, k) * gy + y] = sum_i conj(V_m[i][k]) S[r][i][m] for m = 0..nel/2;
// each V entry is loaded once for the R rows.
template <int R>
__global__ void __launch_bounds__(kBlochThreads, 8) bloch_x_forward(BlochDir bx, int gy,
                                                                 const double* __restrict__ F,
                                                                 double2* __restrict__ xh) {
  extern __shared__ double2 bsm[];
  const int nel = bx.nel, p = bx.p, gx = nel * p, mx = nel / 2 + 1;
  const int y0 = blockIdx.x * R;
  double2* S = bsm;  // [R][p][nel]
  double2* tw = bsm + R * gx;  // [nel/2]
  for (int t = threadIdx.x; t < nel / 2; t += blockDim.x) tw[t] = bx.tw[t];
  for (int t = threadIdx.x; t < R * gx; t += blockDim.x) {
    const int r = t / gx, u = t - r * gx, e = u / p, i = u - e * p;
    const int y = y0 + r;
    S[(r * p + i) * nel + bitrev(e, bx.logn)] =
        make_double2(y < gy ? F[(size_t)y * gx + u] : 0.0, 0.0);
  }
  __syncthreads();
  fft_seqs(S, R * p, nel, bx.logn, tw, false);
  // one output (m, k, r) per thread and pass, r fastest (contiguous stores);
  // the p-term sum unrolled to the largest order so that every load is
  // issued before the arithmetic
  for (int o = threadIdx.x; o < mx * p * R; o += blockDim.x) {
    const int c = o / R, r = o - c * R, m = c / p, k = c - m * p;
    const double2* V = bx.V + (size_t)m * p * p + k;
    const double2* Sr = S + (r * p) * nel + m;
    double2 acc = make_double2(0.0, 0.0);
#pragma unroll
    for (int i = 0; i < kBlochMaxP; i++) {
      if (i < p) {
        const double2 t = cmulc(V[i * p], Sr[i * nel]);
        acc.x += t.x;
        acc.y += t.y;
      }
    }
    if (y0 + r < gy) xh[(size_t)c * gy + y0 + r] = acc;
  }
}

// C consecutive x modes c = (m_x, k_x) (modes past the last skipped): their
// columns of the spectral array along y.
template <int C>
__global__ void __launch_bounds__(kBlochThreads, 8) bloch_y_solve(BlochDir bx, BlochDir by, int cols,
                                                               double alpha, double cx, double cy,
                                                               double null_tol, double scale,
                                                               double2* __restrict__ xh) {
  extern __shared__ double2 bsm[];
  const int nel = by.nel, p = by.p, gy = nel * p;
  const int c0 = blockIdx.x * C;
  double2* S = bsm;                // [C][p][nel]
  double2* T = bsm + C * p * nel;  // [C][p][nel]
  double2* tw = T + C * p * nel;   // [nel/2]
  for (int t = threadIdx.x; t < nel / 2; t += blockDim.x) tw[t] = by.tw[t];
  for (int t = threadIdx.x; t < C * gy; t += blockDim.x) {
    const int q = t / gy, u = t - q * gy, e = u / p, i = u - e * p;
    S[(q * p + i) * nel + bitrev(e, by.logn)] =
        c0 + q < cols ? xh[(size_t)(c0 + q) * gy + u] : make_double2(0.0, 0.0);
  }
  __syncthreads();
  fft_seqs(S, C * p, nel, by.logn, tw, false);
  double mux[C];
#pragma unroll
  for (int q = 0; q < C; q++) {
    const int c = min(c0 + q, cols - 1), kx = c % bx.p, mxi = c / bx.p;
    mux[q] = bx.mu[mxi * bx.p + kx];
  }
  // T[q][k][m] = (sum_i conj(V_m[i][k]) S[q][i][m]) / (alpha + cx mu_x + cy mu_y(m, k))
  for (int o = threadIdx.x; o < nel * p * C; o += blockDim.x) {
    const int mk = o / C, q = o - mk * C, m = mk / p, k = mk - m * p;
    const double2* V = by.V + (size_t)m * p * p + k;
    const double2* Sq = S + (q * p) * nel + m;
    double2 acc = make_double2(0.0, 0.0);
#pragma unroll
    for (int i = 0; i < kBlochMaxP; i++) {
      if (i < p) {
        const double2 t = cmulc(V[i * p], Sq[i * nel]);
        acc.x += t.x;
        acc.y += t.y;
      }
    }
    const double d = alpha + cx * mux[q] + cy * by.mu[m * p + k];
    const double f = fabs(d) <= null_tol ? 0.0 : scale / d;
    T[(q * p + k) * nel + m] = make_double2(acc.x * f, acc.y * f);
  }
  __syncthreads();
  // S[q][i][rev(m)] = sum_k V_m[i][k] T[q][k][m], then the inverse FFT over m
  for (int o = threadIdx.x; o < nel * p * C; o += blockDim.x) {
    const int mi = o / C, q = o - mi * C, m = mi / p, i = mi - m * p;
    const double2* V = by.V + (size_t)m * p * p + i * p;
    const double2* Tq = T + (q * p) * nel + m;
    double2 acc = make_double2(0.0, 0.0);
#pragma unroll
    for (int k = 0; k < kBlochMaxP; k++) {
      if (k < p) {
        const double2 t = cmul(V[k], Tq[k * nel]);
        acc.x += t.x;
        acc.y += t.y;
      }
    }
    S[(q * p + i) * nel + bitrev(m, by.logn)] = acc;
  }
  __syncthreads();
  fft_seqs(S, C * p, nel, by.logn, tw, true);
  for (int t = threadIdx.x; t < C * gy; t += blockDim.x) {
    const int q = t / gy, u = t - q * gy, e = u / p, i = u - e * p;
    if (c0 + q < cols) xh[(size_t)(c0 + q) * gy + u] = S[(q * p + i) * nel + e];
  }
}

// R consecutive rows: T[r][i][m] = sum_k V_m[i][k] xh[(m,k) * gy + y] for
// m <= nel/2, the rest by conjugate symmetry, inverse FFT over m, out (+)=
// the real part.
template <int R>
__global__ void __launch_bounds__(kBlochThreads, 8) bloch_x_backward(BlochDir bx, int gy,
                                                                  const double2* __restrict__ xh,
                                                                  double* __restrict__ out,
                                                                  int accumulate) {
  extern __shared__ double2 bsm[];
  const int nel = bx.nel, p = bx.p, gx = nel * p, mx = nel / 2 + 1;
  const int y0 = blockIdx.x * R;
  double2* S = bsm;  // [R][p][nel]
  double2* tw = bsm + R * gx;  // [nel/2]
  for (int t = threadIdx.x; t < nel / 2; t += blockDim.x) tw[t] = bx.tw[t];
  for (int o = threadIdx.x; o < mx * p * R; o += blockDim.x) {
    const int mi = o / R, r = o - mi * R, m = mi / p, i = mi - m * p;
    const double2* V = bx.V + (size_t)m * p * p + i * p;
    const double2* col = xh + (size_t)(m * p) * gy + y0 + r;
    double2 acc = make_double2(0.0, 0.0);
    if (y0 + r < gy) {
#pragma unroll
      for (int k = 0; k < kBlochMaxP; k++) {
        if (k < p) {
          const double2 t = cmul(V[k], col[(size_t)k * gy]);
          acc.x += t.x;
          acc.y += t.y;
        }
      }
    }
    double2* Sr = S + (r * p + i) * nel;
    Sr[bitrev(m, bx.logn)] = acc;
    if (m > 0 && m < nel - m) Sr[bitrev(nel - m, bx.logn)] = make_double2(acc.x, -acc.y);
  }
  __syncthreads();
  fft_seqs(S, R * p, nel, bx.logn, tw, true);
  for (int t = threadIdx.x; t < R * gx; t += blockDim.x) {
    const int r = t / gx, u = t - r * gx, e = u / p, i = u - e * p;
    const int y = y0 + r;
    if (y >= gy) continue;
    const double v = S[(r * p + i) * nel + e].x;
    double* dst = out + (size_t)y * gx + u;
    *dst = accumulate ? *dst + v : v;
  }
}

}  // namespace

size_t bloch_spectrum_elems(const BlochDir& bx, const BlochDir& by) {
  return (size_t)(bx.nel / 2 + 1) * bx.p * by.nel * by.p;
}

cudaError_t launch_bloch_inverse(const BlochDir& bx, const BlochDir& by, double alpha, double cx,
                                 double cy, double null_tol, const double* in, double* out,
                                 bool accumulate, double2* xh, cudaStream_t s) {
  const int gy = by.nel * by.p, cols = (bx.nel / 2 + 1) * bx.p;
  // one row (x passes) or one x mode (y pass) per block: the passes are
  // latency-bound, and one block per row keeps every SM's warp slots filled
  const size_t smx = sizeof(double2) * ((size_t)bx.p * bx.nel + bx.nel / 2 + 1);
  const size_t smy = sizeof(double2) * (2 * (size_t)by.p * by.nel + by.nel / 2 + 1);
  if (smx > 48 * 1024 || smy > 48 * 1024) return cudaErrorInvalidValue;
  const double scale = 1.0 / ((double)bx.nel * by.nel);
  bloch_x_forward<1><<<gy, kBlochThreads, smx, s>>>(bx, gy, in, xh);
  bloch_y_solve<1><<<cols, kBlochThreads, smy, s>>>(bx, by, cols, alpha, cx, cy, null_tol, scale,
                                                    xh);
  bloch_x_backward<1><<<gy, kBlochThreads, smx, s>>>(bx, gy, xh, out, accumulate ? 1 : 0);
  return cudaGetLastError();
}

}  // namespace seg
