// Fast diagonalization (FDM) solver pieces for SE's Helmholtz/Poisson
// operator, sm_100a.
//
// On SE's meshes the assembled operator is a sum of Kronecker products of
// 1-D assembled operators (see linsys.cu):
//     A = alpha W_y(x)W_x + beta_x W_y(x)K_x + beta_y K_y(x)W_x
// acting on the unknowns arranged as a G_y x G_x array U (row = y). With the
// generalised eigenvectors S (S^T K S = Lambda, S^T W S = I) of each 1-D pair,
//     S_y^T A(U) S_x = D o (S_y^T U S_x),  D_ij = alpha + beta_x lx_j + beta_y ly_i,
// so A^{-1} F = S_y [(S_y^T F S_x) / D] S_x^T: four dense GEMMs and one
// pointwise division (Lynch, Rice and Thomas, 1964). The transforms are
// exact for every boundary configuration SE builds (periodic directions,
// Dirichlet or natural ends), in both the reference's Laplacian scaling and
// the true-Jacobian one.
//
// This file holds the pointwise kernels around the GEMMs: the spectral
// division (zeroing a null mode), precision conversions with a scale, the
// FP64 residual r = b - A x, the weighted residual norms and the update
// x += d.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "common.cuh"
#include "fdm_ctl.cuh"

namespace seg {
namespace {

// V (column-major G_x x G_y, i = x mode, j = y mode) /= alpha + bx lx_i + by ly_j.
template <class T>
__global__ void spectral_divide_kernel(T* __restrict__ v, int gx, int gy,
                                       const double* __restrict__ lx,
                                       const double* __restrict__ ly, double alpha, double bx,
                                       double by, double null_tol) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y;
  if (i >= gx) return;
  const double d = alpha + bx * lx[i] + by * ly[j];
  const size_t k = (size_t)j * gx + i;
  const double val = (double)v[k];
  v[k] = (T)(fabs(d) <= null_tol ? 0.0 : val / d);
}

// y = x / max|x| in low precision (max from device memory).
template <class T>
__global__ void to_low_kernel(const double* __restrict__ x, T* __restrict__ y, size_t n,
                              const double* __restrict__ mx) {
  const double m = *mx;
  const double scale = m > 0.0 ? 1.0 / m : 0.0;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n;
       k += (size_t)gridDim.x * blockDim.x)
    y[k] = (T)(x[k] * scale);
}

// x += y * max (undoing the scale of to_low).
template <class T>
__global__ void add_low_kernel(double* __restrict__ x, const T* __restrict__ y, size_t n,
                               const double* __restrict__ mx) {
  const double m = *mx;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n;
       k += (size_t)gridDim.x * blockDim.x)
    x[k] += (double)y[k] * m;
}

// ------------------------------------------------- refinement loop control --
__global__ void fdm_init_kernel(const FdmParams* __restrict__ p, FdmState* __restrict__ st,
                                const double* __restrict__ res, cudaGraphConditionalHandle h) {
  fdm_init_state(p, st, res[0], h);
}

__global__ void fdm_check_kernel(const FdmParams* __restrict__ p, FdmState* __restrict__ st,
                                 const double* __restrict__ res, cudaGraphConditionalHandle h) {
  fdm_check_state(p, st, res[0], h);
}

// Fixed-order block reduction of one sum (256 threads); result in thread 0.
__device__ __forceinline__ double block_sum(double v) {
  __shared__ double sm[8];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    v = threadIdx.x < 8 ? sm[threadIdx.x] : 0.0;
#pragma unroll
    for (int o = 4; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  }
  return v;
}

// Per-block partial sums over k of (w_k r_k)^2, or of r_k w_k r_k when
// natural != 0 (w = dinv; w == nullptr means w = 1), and of r_k^2;
// partial[2*block].
__global__ void __launch_bounds__(256) norm_partials_kernel(const double* __restrict__ r,
                                                            const double* __restrict__ w, size_t n,
                                                            int natural,
                                                            double* __restrict__ partial) {
  double s0 = 0.0, s1 = 0.0;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n;
       k += (size_t)gridDim.x * blockDim.x) {
    const double v = r[k];
    const double z = w ? v * w[k] : v;
    s0 = fma(z, natural ? v : z, s0);
    s1 = fma(v, v, s1);
  }
  s0 = block_sum(s0);
  __syncthreads();
  s1 = block_sum(s1);
  if (threadIdx.x == 0) {
    partial[2 * blockIdx.x] = s0;
    partial[2 * blockIdx.x + 1] = s1;
  }
}
__global__ void __launch_bounds__(256) norm_final_kernel(const double* __restrict__ partial, int np,
                                                         double* __restrict__ out) {
  double s0 = 0.0, s1 = 0.0;
  for (int k = threadIdx.x; k < np; k += blockDim.x) {
    s0 += partial[2 * k];
    s1 += partial[2 * k + 1];
  }
  s0 = block_sum(s0);
  __syncthreads();
  s1 = block_sum(s1);
  if (threadIdx.x == 0) {
    out[0] = s0;
    out[1] = s1;
  }
}

// Max-abs of a vector, deterministic two-pass (for the low-precision scale).
__global__ void __launch_bounds__(256) maxabs_partials_kernel(const double* __restrict__ x, size_t n,
                                                              double* __restrict__ partial) {
  double m = 0.0;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n;
       k += (size_t)gridDim.x * blockDim.x)
    m = fmax(m, fabs(x[k]));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
  __shared__ double sm[8];
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < 8; w++) m = fmax(m, sm[w]);
    partial[blockIdx.x] = m;
  }
}
__global__ void maxabs_final_kernel(const double* __restrict__ partial, int np, double* out) {
  double m = 0.0;
  for (int k = threadIdx.x; k < np; k += 32) m = fmax(m, partial[k]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
  if (threadIdx.x == 0) *out = m;
}

// r = b - y (y = A x from the operator kernel)
__global__ void sub_kernel(const double* __restrict__ b, const double* __restrict__ y,
                           double* __restrict__ r, size_t n) {
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n;
       k += (size_t)gridDim.x * blockDim.x)
    r[k] = b[k] - y[k];
}

// x -= mean(x) with the mean from a precomputed sum (null-space removal).
__global__ void sub_mean_kernel(double* __restrict__ x, size_t n, const double* __restrict__ sum) {
  const double m = sum[0] / (double)n;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n;
       k += (size_t)gridDim.x * blockDim.x)
    x[k] -= m;
}
__global__ void __launch_bounds__(256) sum_partials_kernel(const double* __restrict__ x, size_t n,
                                                           double* __restrict__ partial) {
  double s = 0.0;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n;
       k += (size_t)gridDim.x * blockDim.x)
    s += x[k];
  s = block_sum(s);
  if (threadIdx.x == 0) partial[2 * blockIdx.x] = s, partial[2 * blockIdx.x + 1] = 0.0;
}

// Per-block partial sums of f and of d = 1 / dinv (the Jacobi diagonal).
__global__ void __launch_bounds__(256) null_partials_kernel(const double* __restrict__ f,
                                                            const double* __restrict__ dinv,
                                                            size_t n, double* __restrict__ partial) {
  double s0 = 0.0, s1 = 0.0;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n;
       k += (size_t)gridDim.x * blockDim.x) {
    s0 += f[k];
    s1 += 1.0 / dinv[k];
  }
  s0 = block_sum(s0);
  __syncthreads();
  s1 = block_sum(s1);
  if (threadIdx.x == 0) {
    partial[2 * blockIdx.x] = s0;
    partial[2 * blockIdx.x + 1] = s1;
  }
}
// f -= (sum f / sum d) d
__global__ void null_project_kernel(double* __restrict__ f, const double* __restrict__ dinv,
                                    size_t n, const double* __restrict__ sum2) {
  const double c = sum2[0] / sum2[1];
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n;
       k += (size_t)gridDim.x * blockDim.x)
    f[k] -= c / dinv[k];
}

__global__ void invert_kernel(double* __restrict__ x, size_t n) {
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n;
       k += (size_t)gridDim.x * blockDim.x)
    x[k] = 1.0 / x[k];
}

// C = A^T (Bh + Bl) for n x n row-major matrices, every product and sum in
// double-double (TwoProd by FMA, TwoSum), the result returned as the pair
// Ch + Cl. Set-up only: the residuals of the eigenvector refinement, whose
// entries are differences far below the operands' size. Bl may be null.
__global__ void __launch_bounds__(256) dd_gemm_tn_kernel(int n, const double* __restrict__ A,
                                                         const double* __restrict__ Bh,
                                                         const double* __restrict__ Bl,
                                                         double* __restrict__ Ch,
                                                         double* __restrict__ Cl) {
  __shared__ double as[16][17], bh[16][17], bl[16][17];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int i0 = blockIdx.y * 16, j0 = blockIdx.x * 16;
  const int i = i0 + ty, j = j0 + tx;
  double sh = 0.0, sl = 0.0;
  for (int k0 = 0; k0 < n; k0 += 16) {
    const int k = k0 + ty;
    const bool kr = k < n;
    as[ty][tx] = (kr && i0 + tx < n) ? A[(size_t)k * n + i0 + tx] : 0.0;
    bh[ty][tx] = (kr && j < n) ? Bh[(size_t)k * n + j] : 0.0;
    bl[ty][tx] = (Bl && kr && j < n) ? Bl[(size_t)k * n + j] : 0.0;
    __syncthreads();
#pragma unroll 4
    for (int kk = 0; kk < 16; kk++) {
      const double a = as[kk][ty];
      dd_fma(sh, sl, a, bh[kk][tx]);
      sl = fma(a, bl[kk][tx], sl);
    }
    __syncthreads();
  }
  if (i < n && j < n) {
    double s, e;
    two_sum(sh, sl, s, e);
    Ch[(size_t)i * n + j] = s;
    Cl[(size_t)i * n + j] = e;
  }
}

// y = a y + b x (a == 0 does not read y)
__global__ void axpby_kernel(double* __restrict__ y, double a, double b,
                             const double* __restrict__ x, size_t n) {
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n;
       k += (size_t)gridDim.x * blockDim.x)
    y[k] = a == 0.0 ? b * x[k] : fma(a, y[k], b * x[k]);
}

int blocks_for(size_t n) {
  size_t b = (n + 255) / 256;
  return (int)(b < 1184 ? (b < 1 ? 1 : b) : 1184);
}

}  // namespace

cudaError_t launch_spectral_divide(int prec, void* v, int gx, int gy, const double* lx,
                                   const double* ly, double alpha, double bx, double by,
                                   double null_tol, cudaStream_t s) {
  dim3 grid((gx + 255) / 256, gy);
  if (prec == 0)
    spectral_divide_kernel<double><<<grid, 256, 0, s>>>((double*)v, gx, gy, lx, ly, alpha, bx, by,
                                                        null_tol);
  else if (prec == 1)
    spectral_divide_kernel<float><<<grid, 256, 0, s>>>((float*)v, gx, gy, lx, ly, alpha, bx, by,
                                                       null_tol);
  else
    spectral_divide_kernel<__nv_bfloat16><<<grid, 256, 0, s>>>((__nv_bfloat16*)v, gx, gy, lx, ly,
                                                               alpha, bx, by, null_tol);
  return cudaGetLastError();
}

cudaError_t launch_to_low(int prec, const double* x, void* y, size_t n, const double* mx,
                          cudaStream_t s) {
  if (prec == 1)
    to_low_kernel<float><<<blocks_for(n), 256, 0, s>>>(x, (float*)y, n, mx);
  else
    to_low_kernel<__nv_bfloat16><<<blocks_for(n), 256, 0, s>>>(x, (__nv_bfloat16*)y, n, mx);
  return cudaGetLastError();
}

cudaError_t launch_add_low(int prec, double* x, const void* y, size_t n, const double* mx,
                           cudaStream_t s) {
  if (prec == 1)
    add_low_kernel<float><<<blocks_for(n), 256, 0, s>>>(x, (const float*)y, n, mx);
  else
    add_low_kernel<__nv_bfloat16><<<blocks_for(n), 256, 0, s>>>(x, (const __nv_bfloat16*)y, n, mx);
  return cudaGetLastError();
}

cudaError_t launch_fdm_init(const FdmParams* p, FdmState* st, const double* res,
                            cudaGraphConditionalHandle h, cudaStream_t s) {
  fdm_init_kernel<<<1, 1, 0, s>>>(p, st, res, h);
  return cudaGetLastError();
}

cudaError_t launch_fdm_check(const FdmParams* p, FdmState* st, const double* res,
                             cudaGraphConditionalHandle h, cudaStream_t s) {
  fdm_check_kernel<<<1, 1, 0, s>>>(p, st, res, h);
  return cudaGetLastError();
}

cudaError_t launch_norms(const double* r, const double* w, size_t n, int natural, double* partial,
                         int npart, double* out2, cudaStream_t s) {
  int b = blocks_for(n);
  if (b > npart) b = npart;
  norm_partials_kernel<<<b, 256, 0, s>>>(r, w, n, natural, partial);
  norm_final_kernel<<<1, 256, 0, s>>>(partial, b, out2);
  return cudaGetLastError();
}

cudaError_t launch_dd_gemm_tn(int n, const double* A, const double* Bh, const double* Bl,
                              double* Ch, double* Cl, cudaStream_t s) {
  if (n <= 0) return cudaErrorInvalidValue;
  const dim3 grid((n + 15) / 16, (n + 15) / 16);
  dd_gemm_tn_kernel<<<grid, 256, 0, s>>>(n, A, Bh, Bl, Ch, Cl);
  return cudaGetLastError();
}

cudaError_t launch_axpby(double* y, double a, double b, const double* x, size_t n,
                         cudaStream_t s) {
  axpby_kernel<<<blocks_for(n), 256, 0, s>>>(y, a, b, x, n);
  return cudaGetLastError();
}

cudaError_t launch_invert(double* x, size_t n, cudaStream_t s) {
  invert_kernel<<<blocks_for(n), 256, 0, s>>>(x, n);
  return cudaGetLastError();
}

cudaError_t launch_norm_final(const double* partial, int np, double* out2, cudaStream_t s) {
  norm_final_kernel<<<1, 256, 0, s>>>(partial, np, out2);
  return cudaGetLastError();
}

cudaError_t launch_maxabs(const double* x, size_t n, double* partial, int npart, double* out,
                          cudaStream_t s) {
  int b = blocks_for(n);
  if (b > npart) b = npart;
  maxabs_partials_kernel<<<b, 256, 0, s>>>(x, n, partial);
  maxabs_final_kernel<<<1, 32, 0, s>>>(partial, b, out);
  return cudaGetLastError();
}

cudaError_t launch_sub(const double* b, const double* y, double* r, size_t n, cudaStream_t s) {
  sub_kernel<<<blocks_for(n), 256, 0, s>>>(b, y, r, n);
  return cudaGetLastError();
}

cudaError_t launch_remove_mean(double* x, size_t n, double* partial, int npart, double* sum2,
                               cudaStream_t s) {
  int b = blocks_for(n);
  if (b > npart) b = npart;
  sum_partials_kernel<<<b, 256, 0, s>>>(x, n, partial);
  norm_final_kernel<<<1, 256, 0, s>>>(partial, b, sum2);
  sub_mean_kernel<<<blocks_for(n), 256, 0, s>>>(x, n, sum2);
  return cudaGetLastError();
}

cudaError_t launch_project_null(double* f, const double* dinv, size_t n, double* partial,
                                int npart, double* sum2, cudaStream_t s) {
  int b = blocks_for(n);
  if (b > npart) b = npart;
  null_partials_kernel<<<b, 256, 0, s>>>(f, dinv, n, partial);
  norm_final_kernel<<<1, 256, 0, s>>>(partial, b, sum2);
  null_project_kernel<<<blocks_for(n), 256, 0, s>>>(f, dinv, n, sum2);
  return cudaGetLastError();
}

}  // namespace seg
