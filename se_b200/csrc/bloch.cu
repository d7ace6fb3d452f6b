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
// registers a thread (8 blocks per SM), the order a template parameter (the
// p-term sums unrolled, their loads issued together) and the twiddles in
// shared memory.
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

// In-place radix-2 FFTs of length n = 2^logn on NSEQ sequences S[s][0..n)
// (stride n), input in bit-reversed order, output in natural order;
// inverse: conjugate twiddles (tw in shared memory). Unnormalised.
template <int NSEQ>
__device__ __forceinline__ void fft_seqs(double2* S, int n, int logn, const double2* tw,
                                         bool inverse) {
  const int hn = n >> 1, nb = NSEQ * hn;
  for (int s = 1; s <= logn; s++) {
    const int half = 1 << (s - 1), step = n >> s;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) {
      const int q = b >> (logn - 1), j = b & (hn - 1);
      const int pos = j & (half - 1), k0 = ((j >> (s - 1)) << s) + pos, k1 = k0 + half;
      double2* x = S + q * n;
      double2 w = tw[pos * step];
      if (inverse) w.y = -w.y;
      const double2 u = x[k0], v = cmul(x[k1], w);
      x[k0] = make_double2(u.x + v.x, u.y + v.y);
      x[k1] = make_double2(u.x - v.x, u.y - v.y);
    }
    __syncthreads();
  }
}

__device__ __forceinline__ void load_twiddles(double2* tw, const double2* g, int hn) {
  for (int t = threadIdx.x; t < hn; t += blockDim.x) tw[t] = g[t];
}

// Row y = blockIdx.x of the real G_y x G_x array F: S[i][m] =
// sum_e F(e, i) e^{-i th_m e}, then xh[(m, k) * gy + y] =
// sum_i conj(V_m[i][k]) S[i][m] for m = 0..nel/2. With a gate whose reason
// is already set (a refinement loop whose initial test decided), F is read
// as zero, so that the inverse adds nothing.
template <int P>
__global__ void __launch_bounds__(kBlochThreads, 8) bloch_x_forward(BlochDir bx, int gy,
                                                                    const double* __restrict__ F,
                                                                    double2* __restrict__ xh,
                                                                    const FdmState* gate) {
  extern __shared__ double2 bsm[];
  const int nel = bx.nel, logn = bx.logn, gx = nel * P, mx = nel / 2 + 1;
  const int y = blockIdx.x;
  double2* S = bsm;            // [P][nel]
  double2* tw = bsm + P * nel;  // [nel/2]
  load_twiddles(tw, bx.tw, nel >> 1);
  const bool closed = gate && *(volatile const int*)&gate->reason != 0;
  for (int t = threadIdx.x; t < gx; t += blockDim.x) {
    const int e = t / P, i = t - e * P;
    S[i * nel + bitrev(e, logn)] = make_double2(closed ? 0.0 : F[(size_t)y * gx + t], 0.0);
  }
  __syncthreads();
  fft_seqs<P>(S, nel, logn, tw, false);
  for (int o = threadIdx.x; o < mx * P; o += blockDim.x) {
    const int m = o / P, k = o - m * P;
    const double2* V = bx.V + (size_t)m * P * P + k;
    double2 vv[P];
#pragma unroll
    for (int i = 0; i < P; i++) vv[i] = V[i * P];
    double2 acc = make_double2(0.0, 0.0);
#pragma unroll
    for (int i = 0; i < P; i++) {
      const double2 t = cmulc(vv[i], S[i * nel + m]);
      acc.x += t.x;
      acc.y += t.y;
    }
    xh[(size_t)o * gy + y] = acc;
  }
}

// x mode c = blockIdx.x = (m_x, k_x): its column of the spectral array along y.
template <int P>
__global__ void __launch_bounds__(kBlochThreads, 8) bloch_y_solve(BlochDir bx, BlochDir by,
                                                                  double alpha, double cx,
                                                                  double cy, double null_tol,
                                                                  double scale,
                                                                  double2* __restrict__ xh) {
  extern __shared__ double2 bsm[];
  const int nel = by.nel, logn = by.logn, gy = nel * P;
  const int c = blockIdx.x;
  double2* S = bsm;            // [P][nel]
  double2* T = bsm + P * nel;  // [P][nel]
  double2* tw = T + P * nel;   // [nel/2]
  load_twiddles(tw, by.tw, nel >> 1);
  double2* col = xh + (size_t)c * gy;
  for (int t = threadIdx.x; t < gy; t += blockDim.x) {
    const int e = t / P, i = t - e * P;
    S[i * nel + bitrev(e, logn)] = col[t];
  }
  __syncthreads();
  fft_seqs<P>(S, nel, logn, tw, false);
  const double mux = bx.mu[c];  // mu is [m][k]: the x mode's index is c
  // T[k][m] = (sum_i conj(V_m[i][k]) S[i][m]) / (alpha + cx mu_x + cy mu_y(m, k))
  for (int o = threadIdx.x; o < nel * P; o += blockDim.x) {
    const int m = o / P, k = o - m * P;
    const double2* V = by.V + (size_t)m * P * P + k;
    double2 vv[P];
#pragma unroll
    for (int i = 0; i < P; i++) vv[i] = V[i * P];
    double2 acc = make_double2(0.0, 0.0);
#pragma unroll
    for (int i = 0; i < P; i++) {
      const double2 t = cmulc(vv[i], S[i * nel + m]);
      acc.x += t.x;
      acc.y += t.y;
    }
    const double d = alpha + cx * mux + cy * by.mu[o];
    const double f = fabs(d) <= null_tol ? 0.0 : scale / d;
    T[k * nel + m] = make_double2(acc.x * f, acc.y * f);
  }
  __syncthreads();
  // S[i][rev(m)] = sum_k V_m[i][k] T[k][m], then the inverse FFT over m
  for (int o = threadIdx.x; o < nel * P; o += blockDim.x) {
    const int m = o / P, i = o - m * P;
    const double2* V = by.V + (size_t)m * P * P + i * P;
    double2 vv[P];
#pragma unroll
    for (int k = 0; k < P; k++) vv[k] = V[k];
    double2 acc = make_double2(0.0, 0.0);
#pragma unroll
    for (int k = 0; k < P; k++) {
      const double2 t = cmul(vv[k], T[k * nel + m]);
      acc.x += t.x;
      acc.y += t.y;
    }
    S[i * nel + bitrev(m, logn)] = acc;
  }
  __syncthreads();
  fft_seqs<P>(S, nel, logn, tw, true);
  for (int t = threadIdx.x; t < gy; t += blockDim.x) {
    const int e = t / P, i = t - e * P;
    col[t] = S[i * nel + e];
  }
}

// Row y = blockIdx.x: T[i][m] = sum_k V_m[i][k] xh[(m,k) * gy + y] for
// m <= nel/2, the rest by conjugate symmetry, inverse FFT over m, out (+)=
// the real part.
template <int P>
__global__ void __launch_bounds__(kBlochThreads, 8) bloch_x_backward(BlochDir bx, int gy,
                                                                     const double2* __restrict__ xh,
                                                                     double* __restrict__ out,
                                                                     int accumulate) {
  extern __shared__ double2 bsm[];
  const int nel = bx.nel, logn = bx.logn, gx = nel * P, mx = nel / 2 + 1;
  const int y = blockIdx.x;
  double2* S = bsm;            // [P][nel]
  double2* tw = bsm + P * nel;  // [nel/2]
  load_twiddles(tw, bx.tw, nel >> 1);
  for (int o = threadIdx.x; o < mx * P; o += blockDim.x) {
    const int m = o / P, i = o - m * P;
    const double2* V = bx.V + (size_t)m * P * P + i * P;
    const double2* col = xh + (size_t)(m * P) * gy + y;
    double2 vv[P], xv[P];
#pragma unroll
    for (int k = 0; k < P; k++) {
      vv[k] = V[k];
      xv[k] = col[(size_t)k * gy];
    }
    double2 acc = make_double2(0.0, 0.0);
#pragma unroll
    for (int k = 0; k < P; k++) {
      const double2 t = cmul(vv[k], xv[k]);
      acc.x += t.x;
      acc.y += t.y;
    }
    S[i * nel + bitrev(m, logn)] = acc;
    if (m > 0 && m < nel - m) S[i * nel + bitrev(nel - m, logn)] = make_double2(acc.x, -acc.y);
  }
  __syncthreads();
  fft_seqs<P>(S, nel, logn, tw, true);
  for (int t = threadIdx.x; t < gx; t += blockDim.x) {
    const int e = t / P, i = t - e * P;
    const double v = S[i * nel + e].x;
    double* dst = out + (size_t)y * gx + t;
    *dst = accumulate ? *dst + v : v;
  }
}

template <int P>
cudaError_t bloch_run(const BlochDir& bx, const BlochDir& by, double alpha, double cx, double cy,
                      double null_tol, const double* in, double* out, bool accumulate,
                      double2* xh, const FdmState* gate, cudaStream_t s) {
  const int gy = by.nel * P, cols = (bx.nel / 2 + 1) * P;
  const size_t smx = sizeof(double2) * ((size_t)P * bx.nel + bx.nel / 2 + 1);
  const size_t smy = sizeof(double2) * (2 * (size_t)P * by.nel + by.nel / 2 + 1);
  if (smx > 48 * 1024 || smy > 48 * 1024) return cudaErrorInvalidValue;
  bloch_x_forward<P><<<gy, kBlochThreads, smx, s>>>(bx, gy, in, xh, gate);
  bloch_y_solve<P><<<cols, kBlochThreads, smy, s>>>(bx, by, alpha, cx, cy, null_tol,
                                                    1.0 / ((double)bx.nel * by.nel), xh);
  bloch_x_backward<P><<<gy, kBlochThreads, smx, s>>>(bx, gy, xh, out, accumulate ? 1 : 0);
  return cudaGetLastError();
}

}  // namespace

size_t bloch_spectrum_elems(const BlochDir& bx, const BlochDir& by) {
  return (size_t)(bx.nel / 2 + 1) * bx.p * by.nel * by.p;
}

// One row (x passes) or one x mode (y pass) per block: the passes are
// latency-bound, and one block per row keeps every SM's warp slots filled.
cudaError_t launch_bloch_inverse(const BlochDir& bx, const BlochDir& by, double alpha, double cx,
                                 double cy, double null_tol, const double* in, double* out,
                                 bool accumulate, double2* xh, const FdmState* gate,
                                 cudaStream_t s) {
  if (bx.p != by.p) return cudaErrorInvalidValue;
#define SE_BLOCH_P(n) \
  case n:             \
    return bloch_run<n>(bx, by, alpha, cx, cy, null_tol, in, out, accumulate, xh, gate, s);
  switch (bx.p) {
    SE_BLOCH_P(2) SE_BLOCH_P(3) SE_BLOCH_P(4) SE_BLOCH_P(5) SE_BLOCH_P(6) SE_BLOCH_P(7)
    SE_BLOCH_P(8) SE_BLOCH_P(9) SE_BLOCH_P(10) SE_BLOCH_P(11) SE_BLOCH_P(12)
    default:
      return cudaErrorInvalidValue;
  }
#undef SE_BLOCH_P
}

}  // namespace seg
