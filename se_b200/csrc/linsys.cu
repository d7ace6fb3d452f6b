// Matrix-free Helmholtz/Poisson operator and a persistent, deterministic
// Jacobi-preconditioned CG for sm_100a.
//
// Operator. SE assembles A = c*Mass + s*Laplacian element by element into a
// PETSc AIJ matrix (src/base/Matrix.cpp:63-149, src/base/Operator.cpp:63-84,
// 157-177). On SE's meshes every element is the same axis-aligned rectangle
// (src/base/Mesh.cpp:17-84) and the GLL mass matrix is diagonal, so the
// assembled operator is a sum of Kronecker products of 1-D assembled
// operators:
//     A = alpha (W (x) W) + beta_x (Kx (x) W) + beta_y (W (x) Ky)
// with Kx/Ky the assembled 1-D reference stiffness (Kh = D^T diag(w) D) and
// W the assembled 1-D GLL weights. Applying it is a sum-factorised
// contraction along rows and along columns of the unknown grid: at most
// 2N+1 taps per direction, 16 bytes of HBM traffic per unknown in FP64.
// The gather-scatter (direct stiffness summation) is implicit: every output
// unknown sums its own row of the assembled 1-D operators in a fixed order,
// so the result is deterministic and needs no atomics.
//
// The persistent CG that drives this operator is in cg.cu.
#include <algorithm>

#include "common.cuh"
#include "fdm_ctl.cuh"

namespace seg {
namespace {

// Fold a vertex index onto its periodic partner.
__device__ __forceinline__ int fold(const Dir& d, int g) {
  return (d.periodic && g == d.nV - 1) ? 0 : g;
}
__device__ __forceinline__ bool unknown(const Dir& d, int g) { return g >= d.lo && g < d.hi; }

// Assembled 1-D GLL weight of vertex g.
__device__ __forceinline__ double wsum(const OpDev& op, const Dir& d, int g) {
  int e = g / d.N, a = g - e * d.N;
  double s = 0.0;
  if (e < d.nE) s += op.w[a];
  if (a == 0 && (e > 0 || d.periodic)) s += op.w[d.N];
  return s;
}
// Assembled 1-D diagonal of vertex g for the element matrix M (Kh, Sv, Tv).
__device__ __forceinline__ double kdiag(const double* M, const Dir& d, int g) {
  const int n = d.N + 1;
  int e = g / d.N, a = g - e * d.N;
  double s = 0.0;
  if (e < d.nE) s += M[a * n + a];
  if (a == 0 && (e > 0 || d.periodic)) s += M[d.N * n + d.N];
  return s;
}
// Row g of the assembled 1-D stiffness applied to val(vertex): the row of
// element e = g/N at local a, plus the last row of element e-1 when g is the
// element's left end. Dirichlet vertices contribute only when the caller's
// val() returns them.
template <class F>
__device__ __forceinline__ double krow(const OpDev& op, const Dir& d, int g, const F& val) {
  const int N = d.N, n = N + 1;
  int e = g / N, a = g - e * N;
  double s = 0.0;
  if (e < d.nE) {
    const double* k = op.Kh + a * n;
    const int g0 = e * N;
    for (int b = 0; b < n; b++) s = fma(k[b], val(fold(d, g0 + b)), s);
  }
  if (a == 0 && (e > 0 || d.periodic)) {
    const double* k = op.Kh + N * n;
    const int g0 = (e > 0 ? e - 1 : d.nE - 1) * N;
    for (int b = 0; b < n; b++) s = fma(k[b], val(fold(d, g0 + b)), s);
  }
  return s;
}

__device__ __forceinline__ double diag_at(const OpDev& op, int gx, int gy) {
  const double wx = wsum(op, op.d[0], gx), wy = wsum(op, op.d[1], gy);
  const double d = op.alpha * wx * wy + op.beta[0] * kdiag(op.Kh, op.d[0], gx) * wy +
                   op.beta[1] * wx * kdiag(op.Kh, op.d[1], gy);
  if (op.gamma == 0.0) return d;
  return d + op.gamma * kdiag(op.Sv, op.d[0], gx) * kdiag(op.Tv, op.d[1], gy);
}
// The elements holding vertex g along d: their first vertex and the vertex's
// local index in each (at most two).
__device__ __forceinline__ int elems_of(const Dir& d, int g, int* g0, int* loc) {
  const int N = d.N, e = g / N, a = g - e * N;
  int k = 0;
  if (e < d.nE) {
    g0[k] = e * N;
    loc[k++] = a;
  }
  if (a == 0 && (e > 0 || d.periodic)) {
    g0[k] = (e > 0 ? e - 1 : d.nE - 1) * N;
    loc[k++] = N;
  }
  return k;
}

__global__ void op_diag_kernel(const OpDev op, double* __restrict__ d) {
  const int ux = blockIdx.x * blockDim.x + threadIdx.x;
  const int uy = blockIdx.y * blockDim.y + threadIdx.y;
  if (ux >= op.G[0] || uy >= op.G[1]) return;
  d[(size_t)uy * op.G[0] + ux] = diag_at(op, ux + op.d[0].lo, uy + op.d[1].lo);
}

// FieldRHS (src/base/RHSOp.cpp:31-50) assembled by Vector::Assemble
// (src/base/Vector.cpp:89-121): each element contributes detJ*w_i*w_j*f at
// its own vertex, so unknown (gx, gy) sums detJ*w*w*f over the vertices that
// map to it (itself, and the periodic duplicates that fold onto it).
__device__ __forceinline__ int contribs(const Dir& d, int g, int* v, int* side) {
  // returns vertices that fold onto g and whether each is an element's left
  // end (0), an interior node (1) or an element's right end (2)
  int e = g / d.N, a = g - e * d.N, k = 0;
  if (a != 0) {
    v[k] = g;
    side[k++] = 1;
    return k;
  }
  if (e < d.nE) {
    v[k] = g;
    side[k++] = 0;
  }
  if (e > 0) {
    v[k] = g;
    side[k++] = 2;
  } else if (d.periodic) {
    v[k] = d.nV - 1;
    side[k++] = 2;
  }
  return k;
}
// FieldRHS + Vector::Assemble at unknown (ux, uy), plus the lifting.
__device__ __forceinline__ double rhs_value(const OpDev& op, const MeshDev& m,
                                           const double* __restrict__ rhs,
                                           const double* __restrict__ lift, int ux, int uy) {
  const Dir &dx = op.d[0], &dy = op.d[1];
  const int gx = ux + dx.lo, gy = uy + dy.lo;
  int vx[2], sx[2], vy[2], sy[2];
  int nx = contribs(dx, gx, vx, sx), ny = contribs(dy, gy, vy, sy);
  const double detj = (0.5 * m.dx[0]) * (0.5 * m.dx[1]);
  const int nvx = m.nVerts[0];
  double s = 0.0;
  for (int b = 0; b < ny; b++) {
    double wy = sy[b] == 1 ? op.w[gy - (gy / dy.N) * dy.N] : (sy[b] == 0 ? op.w[0] : op.w[dy.N]);
    for (int a = 0; a < nx; a++) {
      double wx = sx[a] == 1 ? op.w[gx - (gx / dx.N) * dx.N] : (sx[a] == 0 ? op.w[0] : op.w[dx.N]);
      if (rhs) s += detj * (wx * wy) * rhs[(size_t)vy[b] * nvx + vx[a]];
    }
  }
  const size_t k = (size_t)uy * op.G[0] + ux;
  return s + (lift ? lift[k] : 0.0);
}
__global__ void rhs_assemble_kernel(const OpDev op, const MeshDev m, const double* __restrict__ rhs,
                                    const double* __restrict__ lift, double* __restrict__ f) {
  const int ux = blockIdx.x * blockDim.x + threadIdx.x;
  const int uy = blockIdx.y * blockDim.y + threadIdx.y;
  if (ux >= op.G[0] || uy >= op.G[1]) return;
  f[(size_t)uy * op.G[0] + ux] = rhs_value(op, m, rhs, lift, ux, uy);
}

// Fixed-order sum of two values over a 256-thread block; result in thread 0.
__device__ __forceinline__ void block_sum2_256(double& a, double& b, double (*red)[2]) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_down_sync(0xffffffffu, a, o);
    b += __shfl_down_sync(0xffffffffu, b, o);
  }
  if (lane == 0) {
    red[warp][0] = a;
    red[warp][1] = b;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    a = b = 0.0;
#pragma unroll
    for (int q = 0; q < 8; q++) {
      a += red[q][0];
      b += red[q][1];
    }
  }
}

// The FDM solve's prologue in one launch: the right-hand side f (as
// rhs_assemble_kernel), r = f, x = 0 and per-block partial sums of the
// initial norms (of (w f)^2, or f w f when natural, and of f^2; w == nullptr
// means w = 1); the block that arrives last sums the partials in block order
// and runs the refinement loop's initial test, which sets its condition.
// No block waits for another.
__global__ void __launch_bounds__(256)
    fdm_prologue_kernel(const OpDev op, const MeshDev m, const double* __restrict__ rhs,
                        const double* __restrict__ lift, double* __restrict__ f,
                        double* __restrict__ r, double* __restrict__ x,
                        const double* __restrict__ w, int natural, double* __restrict__ partial,
                        double* __restrict__ res, unsigned* __restrict__ count,
                        const FdmParams* __restrict__ p, FdmState* __restrict__ st,
                        cudaGraphConditionalHandle h) {
  __shared__ double red[8][2];
  __shared__ unsigned last;
  const size_t n = (size_t)op.G[0] * op.G[1];
  double s0 = 0.0, s1 = 0.0;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n;
       k += (size_t)gridDim.x * blockDim.x) {
    const int uy = (int)(k / op.G[0]), ux = (int)(k - (size_t)uy * op.G[0]);
    const double v = rhs_value(op, m, rhs, lift, ux, uy);
    f[k] = v;
    r[k] = v;
    x[k] = 0.0;
    const double z = w ? v * w[k] : v;
    s0 = fma(z, natural ? v : z, s0);
    s1 = fma(v, v, s1);
  }
  block_sum2_256(s0, s1, red);
  if (threadIdx.x == 0) {
    partial[2 * blockIdx.x] = s0;
    partial[2 * blockIdx.x + 1] = s1;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(count, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  s0 = s1 = 0.0;
  for (unsigned k = threadIdx.x; k < gridDim.x; k += blockDim.x) {
    s0 += __ldcg(partial + 2 * k);
    s1 += __ldcg(partial + 2 * k + 1);
  }
  __syncthreads();
  block_sum2_256(s0, s1, red);
  if (threadIdx.x == 0) {
    res[0] = s0;
    res[1] = s1;
    *count = 0u;
    fdm_init_state(p, st, s0, h);
  }
}

// Matrix::Assemble's Dirichlet lifting (src/base/Matrix.cpp:117-140):
// lift = -sum over Dirichlet columns of A[row, col] * u_D(col).
__global__ void lift_kernel(const OpDev op, const MeshDev m, const double* __restrict__ sol,
                            double* __restrict__ lift) {
  const int ux = blockIdx.x * blockDim.x + threadIdx.x;
  const int uy = blockIdx.y * blockDim.y + threadIdx.y;
  if (ux >= op.G[0] || uy >= op.G[1]) return;
  const Dir &dx = op.d[0], &dy = op.d[1];
  const int gx = ux + dx.lo, gy = uy + dy.lo;
  const int nvx = m.nVerts[0];
  const double wx = wsum(op, dx, gx), wy = wsum(op, dy, gy);
  double kx = krow(op, dx, gx, [&](int g) { return unknown(dx, g) ? 0.0 : sol[(size_t)gy * nvx + g]; });
  double ky = krow(op, dy, gy, [&](int g) { return unknown(dy, g) ? 0.0 : sol[(size_t)g * nvx + gx]; });
  double v = op.beta[0] * wy * kx + op.beta[1] * wx * ky;
  if (op.gamma != 0.0) {
    // the SVV element blocks reach every vertex of the elements holding the
    // unknown: the Dirichlet ones (not unknowns after the periodic fold) lift
    const int n = dx.N + 1;
    int x0[2], lx[2], y0[2], ly[2];
    const int nx = elems_of(dx, gx, x0, lx), ny = elems_of(dy, gy, y0, ly);
    double sv = 0.0;
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++)
        for (int b = 0; b < n; b++) {
          const int vy = fold(dy, y0[j] + b);
          double r = 0.0;
          for (int a = 0; a < n; a++) {
            const int vx = fold(dx, x0[i] + a);
            if (unknown(dx, vx) && unknown(dy, vy)) continue;
            r = fma(op.Sv[lx[i] * n + a], sol[(size_t)vy * nvx + vx], r);
          }
          sv = fma(op.Tv[ly[j] * n + b], r, sv);
        }
    v += op.gamma * sv;
  }
  lift[(size_t)uy * op.G[0] + ux] = -v;
}

// Vector::UpdateField (src/base/Vector.cpp:40-61) with the periodic copies.
// dst = src over n2 16-byte pairs and, with an odd count, the last value.
__global__ void __launch_bounds__(256) copy_pairs_kernel(double2* __restrict__ dst,
                                                         const double2* __restrict__ src,
                                                         size_t n2, double* __restrict__ dlast,
                                                         const double* __restrict__ slast) {
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n2;
       k += (size_t)gridDim.x * blockDim.x)
    dst[k] = src[k];
  if (dlast && blockIdx.x == 0 && threadIdx.x == 0) *dlast = *slast;
}

// Also copies a refinement loop's final state st to st_host (a mapped
// page-locked buffer) when both are given: the solve graph's last kernel
// returns the state without a separate copy.
__global__ void update_field_kernel(const OpDev op, const MeshDev m, const double* __restrict__ x,
                                    double* __restrict__ sol, const FdmState* __restrict__ st,
                                    FdmState* st_host) {
  const int ux = blockIdx.x * blockDim.x + threadIdx.x;
  const int uy = blockIdx.y * blockDim.y + threadIdx.y;
  if (st && st_host && ux == 0 && uy == 0) {
    *st_host = *st;
    __threadfence_system();
  }
  if (ux >= op.G[0] || uy >= op.G[1]) return;
  const int gx = ux + op.d[0].lo, gy = uy + op.d[1].lo;
  const int nvx = m.nVerts[0], nvy = m.nVerts[1];
  const double v = x[(size_t)uy * op.G[0] + ux];
  sol[(size_t)gy * nvx + gx] = v;
  const bool cx = op.d[0].periodic && gx == 0, cy = op.d[1].periodic && gy == 0;
  if (cx) sol[(size_t)gy * nvx + nvx - 1] = v;
  if (cy) sol[(size_t)(nvy - 1) * nvx + gx] = v;
  if (cx && cy) sol[(size_t)nvy * nvx - 1] = v;
}

}  // namespace

size_t cg_smem_bytes(int maxN) {
  return sizeof(double) * (size_t)(kCgTileX + 2 * maxN) * (kCgTileY + 2 * maxN);
}

cudaError_t launch_op_diag(const OpDev& op, double* d, cudaStream_t s) {
  dim3 block(32, 8), grid((op.G[0] + 31) / 32, (op.G[1] + 7) / 8);
  op_diag_kernel<<<grid, block, 0, s>>>(op, d);
  return cudaGetLastError();
}
cudaError_t launch_rhs_assemble(const OpDev& op, const MeshDev& m, const double* rhs_vals,
                                const double* lift, double* f, cudaStream_t s) {
  dim3 block(32, 8), grid((op.G[0] + 31) / 32, (op.G[1] + 7) / 8);
  rhs_assemble_kernel<<<grid, block, 0, s>>>(op, m, rhs_vals, lift, f);
  return cudaGetLastError();
}
cudaError_t launch_fdm_prologue(const OpDev& op, const MeshDev& m, const double* rhs_vals,
                                const double* lift, double* f, double* r, double* x,
                                const double* w, int natural, double* partial, int npart,
                                double* res, unsigned* count, const FdmParams* p, FdmState* st,
                                cudaGraphConditionalHandle h, cudaStream_t s) {
  const size_t n = (size_t)op.G[0] * op.G[1];
  if (n == 0 || npart <= 0 || !count) return cudaErrorInvalidValue;
  const int blocks = (int)std::min<size_t>((n + 255) / 256, (size_t)npart);
  fdm_prologue_kernel<<<blocks, 256, 0, s>>>(op, m, rhs_vals, lift, f, r, x, w, natural, partial,
                                             res, count, p, st, h);
  return cudaGetLastError();
}
cudaError_t launch_copy(double* dst, const double* src, size_t n, cudaStream_t s) {
  if (n == 0) return cudaSuccess;
  // a copy kernel over 16-byte pairs when both ends are 16-byte aligned
  // (its launch waits less than the driver's device-to-device copy)
  if (((reinterpret_cast<uintptr_t>(dst) | reinterpret_cast<uintptr_t>(src)) & 15u) != 0)
    return cudaMemcpyAsync(dst, src, sizeof(double) * n, cudaMemcpyDeviceToDevice, s);
  const size_t n2 = n / 2;
  const int blocks = (int)std::min<size_t>(std::max<size_t>((n2 + 255) / 256, 1), 148 * 8);
  copy_pairs_kernel<<<blocks, 256, 0, s>>>(reinterpret_cast<double2*>(dst),
                                           reinterpret_cast<const double2*>(src), n2,
                                           (n & 1) ? dst + n - 1 : nullptr,
                                           (n & 1) ? src + n - 1 : nullptr);
  return cudaGetLastError();
}
cudaError_t launch_lift(const OpDev& op, const MeshDev& m, const double* sol_vals, double* lift,
                        cudaStream_t s) {
  dim3 block(32, 8), grid((op.G[0] + 31) / 32, (op.G[1] + 7) / 8);
  lift_kernel<<<grid, block, 0, s>>>(op, m, sol_vals, lift);
  return cudaGetLastError();
}
cudaError_t launch_update_field(const OpDev& op, const MeshDev& m, const double* x,
                                double* sol_vals, cudaStream_t s, const FdmState* st,
                                FdmState* st_host) {
  dim3 block(32, 8), grid((op.G[0] + 31) / 32, (op.G[1] + 7) / 8);
  update_field_kernel<<<grid, block, 0, s>>>(op, m, x, sol_vals, st, st_host);
  return cudaGetLastError();
}

}  // namespace seg
