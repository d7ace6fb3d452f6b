// Matrix-free operator apply y = A x of SE's assembled Helmholtz/Poisson
// operator on the unknown grid, element-structured, sm_100a.
//
// A = alpha (W_y x W_x) + beta_x (W_y x K_x) + beta_y (K_y x W_x), with K the
// assembled 1-D stiffness and W the assembled 1-D GLL weights (linsys.cu).
// Along one grid row the assembled K_x is the element matrix Kh (order N,
// (N+1) x (N+1)) applied to every element's N+1 nodes, the two contributions
// at a node shared by neighbouring elements summed. A block owns a tile of
// TEX x TEY elements (TEX*N x TEY*N output vertices):
//   0. per-block tables: unknown row/column offsets of the staged vertices
//      and the assembled weights of the tile's rows and columns;
//   1. stages x over the tile plus one element on the left/bottom and one
//      vertex on the right/top (zero where there is no unknown: Dirichlet
//      vertices, outside a non-periodic mesh), all loads issued first;
//   2. rows: the item (row, element k) holds the N+1 values of element k and
//      of its left neighbour in registers and writes the element's first N
//      nodes, O = alpha wx wy u + beta_x wy (Kh u_k + [Kh u_{k-1}]_N at the
//      shared node), with Kh read from the kernel parameters at compile-time
//      indices (constant-bank operands, no loads);
//   3. columns: the item (column, element k) adds beta_y wx (K_y u) the same
//      way and writes y for its N nodes to global memory.
// Every node is produced by one thread in a fixed order of operations, so
// the result does not depend on scheduling. A neighbour element that does
// not exist (non-periodic edge) contributes nothing.
//
// Instantiated for FP64 (x, arithmetic and y in FP64) and for the reduced-
// precision apply (x in BF16 or FP16, operator and arithmetic in FP32, y in
// FP32).
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "common.cuh"

namespace seg {
namespace {

constexpr int kThreads = 256;

template <int N>
struct ATile {
  static constexpr int TEX = 64 / N > 0 ? 64 / N : 1;  // elements per tile
  static constexpr int TEY = 32 / N > 0 ? 32 / N : 1;
  static constexpr int TW = TEX * N, TH = TEY * N;     // output vertices per tile
  static constexpr int UW = TW + N + 1, UH = TH + N + 1;  // staged vertices
  static constexpr int UP = UW | 1;                    // staged row pitch (odd)
  static constexpr int OP = TW + 1;                    // row-phase output pitch
  static constexpr int NU = UH * UP, NO = TH * OP;
  static constexpr int STAGE_ITERS = (UW * UH + kThreads - 1) / kThreads;
  template <class A>
  static constexpr size_t smem() {
    return sizeof(A) * (size_t)(NU + NO + TW + TH) + sizeof(int) * (size_t)(UW + UH);
  }
};

// Operator coefficients in the arithmetic type, passed by value (the kernel
// parameter bank).
template <class A>
struct ApplyOp {
  A Kh[SE_MAXN1 * SE_MAXN1];
  A w[SE_MAXN1];
  A alpha, bx, by;
  Dir dx, dy;
  int G0, G1;
};

__device__ __forceinline__ double to_a(double v, double) { return v; }
__device__ __forceinline__ float to_a(__nv_bfloat16 v, float) { return __bfloat162float(v); }
__device__ __forceinline__ float to_a(__half v, float) { return __half2float(v); }

// Unknown index of vertex g along d (-1: Dirichlet or outside), one wrap for
// periodic directions.
__device__ __forceinline__ int unk(const Dir& d, int g) {
  if (d.periodic) {
    const int L = d.nV - 1;
    if (g < 0)
      g += L;
    else if (g >= L)
      g -= L;
  } else if (g < 0 || g >= d.nV) {
    return -1;
  }
  return (g >= d.lo && g < d.hi) ? g - d.lo : -1;
}

// Assembled 1-D weight of vertex (element e, node a).
template <int N, class A>
__device__ __forceinline__ A wsum(const Dir& d, const A* w, int e, int a) {
  A s = A(0);
  if (e < d.nE) s += w[a];
  if (a == 0 && (e > 0 || d.periodic)) s += w[N];
  return s;
}

template <int N, class TI, class A, class TO>
__global__ void __launch_bounds__(kThreads) apply_tile_kernel(const ApplyOp<A> op,
                                                              const TI* __restrict__ x,
                                                              TO* __restrict__ y) {
  typedef ATile<N> T;
  constexpr int n = N + 1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  A* U = reinterpret_cast<A*>(smem_raw);
  A* O = U + T::NU;
  A* Wx = O + T::NO;  // assembled weights of the tile's columns / rows
  A* Wy = Wx + T::TW;
  int* colu = reinterpret_cast<int*>(Wy + T::TH);  // unknown column of staged column i (-1: none)
  int* rowu = colu + T::UW;                         // unknown row offset of staged row j (-1: none)
  const int gx0 = blockIdx.x * T::TW, gy0 = blockIdx.y * T::TH;
  const int ex0 = gx0 / N, ey0 = gy0 / N;

  // 0. tables
  for (int k = threadIdx.x; k < T::UW + T::UH + T::TW + T::TH; k += kThreads) {
    if (k < T::UW) {
      colu[k] = unk(op.dx, gx0 - N + k);
    } else if (k < T::UW + T::UH) {
      const int uy = unk(op.dy, gy0 - N + (k - T::UW));
      rowu[k - T::UW] = uy < 0 ? -1 : uy * op.G0;
    } else if (k < T::UW + T::UH + T::TW) {
      const int c = k - T::UW - T::UH, kx = c / N;
      Wx[c] = wsum<N>(op.dx, op.w, ex0 + kx, c - kx * N);
    } else {
      const int r = k - T::UW - T::UH - T::TW, ky = r / N;
      Wy[r] = wsum<N>(op.dy, op.w, ey0 + ky, r - ky * N);
    }
  }
  __syncthreads();

  // 1. stage (all loads issued before the stores)
  {
    A v[T::STAGE_ITERS];
#pragma unroll
    for (int s = 0; s < T::STAGE_ITERS; s++) {
      const int k = threadIdx.x + s * kThreads;
      v[s] = A(0);
      if (k < T::UW * T::UH) {
        const int j = k / T::UW, i = k - j * T::UW;
        const int ro = rowu[j], cu = colu[i];
        if (ro >= 0 && cu >= 0) v[s] = to_a(x[(size_t)ro + cu], A(0));
      }
    }
#pragma unroll
    for (int s = 0; s < T::STAGE_ITERS; s++) {
      const int k = threadIdx.x + s * kThreads;
      if (k < T::UW * T::UH) {
        const int j = k / T::UW, i = k - j * T::UW;
        U[j * T::UP + i] = v[s];
      }
    }
  }
  __syncthreads();

  // 2. rows: items (row r, element k); O = alpha wx wy u + beta_x wy (K_x u)
  for (int it = threadIdx.x; it < T::TH * T::TEX; it += kThreads) {
    const int r = it % T::TH, k = it / T::TH;
    const bool own = op.dx.periodic || (ex0 + k < op.dx.nE);
    const bool left = op.dx.periodic || (ex0 + k - 1 >= 0 && ex0 + k - 1 < op.dx.nE);
    const A* u = U + (r + N) * T::UP + k * N;  // left element's node 0
    A ul[n], uo[n];
#pragma unroll
    for (int b = 0; b < n; b++) ul[b] = left ? u[b] : A(0);
#pragma unroll
    for (int b = 0; b < n; b++) uo[b] = own ? u[N + b] : A(0);
    const A wy = Wy[r], sy = op.bx * wy, my = op.alpha * wy;
    A* o = O + r * T::OP + k * N;
#pragma unroll
    for (int a = 0; a < N; a++) {
      A z = A(0);
      if (a == 0) {
#pragma unroll
        for (int b = 0; b < n; b++) z = fma(op.Kh[N * n + b], ul[b], z);
      }
#pragma unroll
      for (int b = 0; b < n; b++) z = fma(op.Kh[a * n + b], uo[b], z);
      o[a] = fma(my * Wx[k * N + a], u[N + a], sy * z);
    }
  }
  __syncthreads();

  // 3. columns: items (column c, element k); y = O + beta_y wx (K_y u)
  for (int it = threadIdx.x; it < T::TW * T::TEY; it += kThreads) {
    const int c = it % T::TW, k = it / T::TW;
    const int gx = gx0 + c;
    if (gx < op.dx.lo || gx >= op.dx.hi) continue;
    const bool own = op.dy.periodic || (ey0 + k < op.dy.nE);
    const bool left = op.dy.periodic || (ey0 + k - 1 >= 0 && ey0 + k - 1 < op.dy.nE);
    const A* u = U + (k * N) * T::UP + (c + N);  // lower element's node 0
    A ul[n], uo[n];
#pragma unroll
    for (int b = 0; b < n; b++) ul[b] = left ? u[b * T::UP] : A(0);
#pragma unroll
    for (int b = 0; b < n; b++) uo[b] = own ? u[(N + b) * T::UP] : A(0);
    const A sx = op.by * Wx[c];
    const int gyk = gy0 + k * N;
#pragma unroll
    for (int a = 0; a < N; a++) {
      A z = A(0);
      if (a == 0) {
#pragma unroll
        for (int b = 0; b < n; b++) z = fma(op.Kh[N * n + b], ul[b], z);
      }
#pragma unroll
      for (int b = 0; b < n; b++) z = fma(op.Kh[a * n + b], uo[b], z);
      const int gy = gyk + a;
      if (gy >= op.dy.lo && gy < op.dy.hi)
        y[(size_t)(gy - op.dy.lo) * op.G0 + (gx - op.dx.lo)] =
            (TO)fma(sx, z, O[(k * N + a) * T::OP + c]);
    }
  }
}

template <int N, class TI, class A, class TO>
cudaError_t launch_tile(const OpDev& od, const TI* x, TO* y, cudaStream_t s) {
  typedef ATile<N> T;
  ApplyOp<A> op;
  for (int k = 0; k < (N + 1) * (N + 1); k++) op.Kh[k] = (A)od.Kh[k];
  for (int k = 0; k <= N; k++) op.w[k] = (A)od.w[k];
  op.alpha = (A)od.alpha;
  op.bx = (A)od.beta[0];
  op.by = (A)od.beta[1];
  op.dx = od.d[0];
  op.dy = od.d[1];
  op.G0 = od.G[0];
  op.G1 = od.G[1];
  constexpr size_t smem = T::template smem<A>();
  static bool attr[64] = {};  // per instantiation and device
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  if (!attr[dev]) {
    e = cudaFuncSetAttribute(apply_tile_kernel<N, TI, A, TO>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    attr[dev] = true;
  }
  const dim3 grid((od.d[0].hi + T::TW - 1) / T::TW, (od.d[1].hi + T::TH - 1) / T::TH);
  apply_tile_kernel<N, TI, A, TO><<<grid, kThreads, smem, s>>>(op, x, y);
  return cudaGetLastError();
}

}  // namespace

#define SE_APPLY_N(n) \
  case n:             \
    return launch_tile<n, double, double, double>(op, x, y, s);
cudaError_t launch_op_apply(const OpDev& op, const double* x, double* y, cudaStream_t s) {
  switch (op.d[0].N) {
    SE_APPLY_N(2) SE_APPLY_N(3) SE_APPLY_N(4) SE_APPLY_N(5) SE_APPLY_N(6) SE_APPLY_N(7)
    SE_APPLY_N(8) SE_APPLY_N(9) SE_APPLY_N(10) SE_APPLY_N(11) SE_APPLY_N(12)
    default:
      return cudaErrorInvalidValue;
  }
}
#undef SE_APPLY_N

#define SE_APPLY_LOW_N(n)                                                                  \
  case n:                                                                                  \
    return fp16 ? launch_tile<n, __half, float, float>(op, (const __half*)x, y, s)         \
                : launch_tile<n, __nv_bfloat16, float, float>(op, (const __nv_bfloat16*)x, y, s);
cudaError_t launch_op_apply_low(const OpDev& op, int fp16, const void* x, float* y, cudaStream_t s) {
  switch (op.d[0].N) {
    SE_APPLY_LOW_N(2) SE_APPLY_LOW_N(3) SE_APPLY_LOW_N(4) SE_APPLY_LOW_N(5) SE_APPLY_LOW_N(6)
    SE_APPLY_LOW_N(7) SE_APPLY_LOW_N(8) SE_APPLY_LOW_N(9) SE_APPLY_LOW_N(10) SE_APPLY_LOW_N(11)
    SE_APPLY_LOW_N(12)
    default:
      return cudaErrorInvalidValue;
  }
}
#undef SE_APPLY_LOW_N

}  // namespace seg
