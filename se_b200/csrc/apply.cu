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
// FP32). In FP64, orders 4 to 8 run the element-factored kernel on the
// FP64 FMA pipes (apply_ef_kernel, at the end of this file) and the other
// orders the same element products on the FP64 tensor cores
// (apply_mma_kernel).
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <cstdint>
#include <cstring>

#include "common.cuh"
#include "fdm_ctl.cuh"

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

// ---------------------------------------------------------------------------
// FP64 apply on the FP64 tensor cores (mma.sync m16n8k8 f64), tiles staged
// by TMA. The 1-D element products are small GEMMs: for element k of a
// tile, the outputs a = 0..N-1 of 16 grid rows are
//     Z (16 x N) = W (16 x 8KS) * B (8KS x N),
// W the staged values of the element's window (its left neighbour's nodes
// and its own: staged columns kN .. kN+2N, padded to 8KS), and
//     B[j][a] = Kh[a][j-N] (own element, j >= N) + [a == 0] Kh[N][j] (left
// element, j <= N), zero in the padding,
// the same matrix for every element and tile, held in registers as MMA
// fragments for the whole kernel. The column direction is the same product
// on the transposed window. At a natural (non-periodic, non-Dirichlet) mesh
// edge the missing neighbour's term at the edge vertex is subtracted.
//
// Persistent blocks take tiles in turn with two shared-memory stages: one
// thread issues the next tile's 2-D TMA load (a UP x UH box of the unknown
// array, its first column rounded down to an even unknown so that the copy
// starts on a 16-byte boundary, out-of-range rows and columns zero-filled)
// while the block computes the current tile. A tile whose staged vertices
// wrap around a periodic direction, or any tile when the unknown array does
// not meet TMA's alignment rules, is staged by ordinary loads instead. Every
// wait on a stage's barrier is bounded; one that gives up sets
// KERR_BARRIER_TIMEOUT in the error word and the tile's result is invalid.
template <int N>
struct MTile {
  typedef ATile<N> T;
  static constexpr int TEX = T::TEX, TEY = T::TEY, TW = T::TW, TH = T::TH;
  static constexpr int KS = (2 * N + 1 + 7) / 8;  // k-steps of the window
  static constexpr int NT = (N + 7) / 8;          // n-tiles of the outputs
  static constexpr int RB = (TH + 15) / 16;       // 16-row blocks
  static constexpr int CB = (TW + 15) / 16;       // 16-column blocks
  static constexpr int cmax(int a, int b) { return a > b ? a : b; }
  // staged rectangle the windows read (the real one plus padding)
  static constexpr int UW = cmax(cmax(T::UW, (TEX - 1) * N + 8 * KS), CB * 16 + N);
  static constexpr int UH = cmax(cmax(T::UH, (TEY - 1) * N + 8 * KS), RB * 16 + N);
  // box width = row pitch: one spare column for the alignment shift, 4 mod 16
  static constexpr int UP = ((UW + 1 + 11) / 16) * 16 + 4;
  static constexpr int OP = TW + 1;
  static constexpr int NU = ((UH * UP * 8 + 127) / 128) * 16;  // doubles per stage (128-byte multiple)
  static constexpr unsigned BOX_BYTES = (unsigned)(UP * UH * 8);
  static constexpr int NO = TH * OP;
  static constexpr size_t SMEM = 128 + 16 + sizeof(double) * (size_t)(2 * NU + NO + TW + TH);
};

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Wait for a barrier phase, at most 2^20 polls; false when the polls ran
// out (the error bit is then set).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity, unsigned* err) {
  for (int it = 0; it < (1 << 20); it++)
    if (mbar_try_wait(bar, parity)) return true;
  atomicOr(err, (unsigned)KERR_BARRIER_TIMEOUT);
  return false;
}
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, "
      "%3}], [%4];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void dmma(double (&c)[4], double a0, double a1, double a2, double a3,
                                     double b0, double b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
      : "d"(a0), "d"(a1), "d"(a2), "d"(a3), "d"(b0), "d"(b1));
}

// Window matrix entry B[j][a].
template <int N>
__device__ __forceinline__ double bwin(const ApplyOp<double>& op, int j, int a) {
  constexpr int n = N + 1;
  if (a >= N || j > 2 * N) return 0.0;
  double v = 0.0;
  if (j >= N) v += op.Kh[a * n + (j - N)];
  if (a == 0 && j <= N) v += op.Kh[N * n + j];
  return v;
}

// Tile t's staged origin in unknown coordinates, and whether TMA can load it.
template <int N>
__device__ __forceinline__ bool tile_tma(const ApplyOp<double>& op, int tma, int tiles_x, int t,
                                         int& xs, int& ys) {
  typedef MTile<N> T;
  const int gx0 = (t % tiles_x) * T::TW, gy0 = (t / tiles_x) * T::TH;
  xs = gx0 - N - op.dx.lo;
  ys = gy0 - N - op.dy.lo;
  if (!tma) return false;
  if (op.dx.periodic && (xs < 0 || xs + ATile<N>::UW > op.G0)) return false;
  if (op.dy.periodic && (ys < 0 || ys + ATile<N>::UH > op.G1)) return false;
  return true;
}

template <int N>
__global__ void __launch_bounds__(kThreads) apply_mma_kernel(const __grid_constant__ CUtensorMap map,
                                                             const ApplyOp<double> op,
                                                             const double* __restrict__ x,
                                                             double* __restrict__ y, int tiles_x,
                                                             int ntiles, int tma,
                                                             unsigned* err) {
  typedef MTile<N> T;
  constexpr int n = N + 1;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* base =
      smem_raw + ((128 - (smem_u32(smem_raw) & 127)) & 127);  // 128-byte aligned stages
  double* Ubuf = reinterpret_cast<double*>(base);                // [2][NU]
  double* O = Ubuf + 2 * T::NU;
  double* Wx = O + T::NO;
  double* Wy = Wx + T::TW;
  uint64_t* bar = reinterpret_cast<uint64_t*>(Wy + T::TH);  // [2]
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, tq = lane & 3;
  if (blockIdx.x >= ntiles) return;

  // B fragments (kept for the whole kernel)
  double bf[T::KS][T::NT][2];
#pragma unroll
  for (int ks = 0; ks < T::KS; ks++)
#pragma unroll
    for (int nt = 0; nt < T::NT; nt++) {
      bf[ks][nt][0] = bwin<N>(op, ks * 8 + tq, nt * 8 + g);
      bf[ks][nt][1] = bwin<N>(op, ks * 8 + tq + 4, nt * 8 + g);
    }

  if (threadIdx.x == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int xs, ys;
    if (tile_tma<N>(op, tma, tiles_x, blockIdx.x, xs, ys)) {
      mbar_expect_tx(&bar[0], T::BOX_BYTES);
      tma_load_2d(Ubuf, &map, xs & ~1, ys, &bar[0]);
    }
  }

  const bool nat_x = !op.dx.periodic, nat_y = !op.dy.periodic;
  const int lastx = op.dx.nV - 1, lasty = op.dy.nV - 1;
  unsigned phase = 0;  // bit s: parity of stage s's next completion
  int i = 0;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x, i++) {
    const int s = i & 1;
    double* U = Ubuf + s * T::NU;
    const int gx0 = (t % tiles_x) * T::TW, gy0 = (t / tiles_x) * T::TH;
    const int ex0 = gx0 / N, ey0 = gy0 / N;
    int xs, ys, off = 0;
    if (tile_tma<N>(op, tma, tiles_x, t, xs, ys)) {
      const bool arrived = mbar_wait_bounded(&bar[s], (phase >> s) & 1u, err);
      // a stage that never arrived: no thread computes on it or issues
      // another load; the block waits (bounded) for the copy still in
      // flight into that stage, so that it does not land after the block
      // has left, and returns with the error bit set
      if (__syncthreads_or(!arrived)) {
        for (int it = 0; it < (1 << 20); it++)
          if (mbar_try_wait(&bar[s], (phase >> s) & 1u)) break;
        return;
      }
      phase ^= 1u << s;
      off = xs & 1;
    } else {
      // ordinary loads: warp w takes staged rows w, w + 8, ...
      typedef ATile<N> R;
      const int vx0 = gx0 - N, vy0 = gy0 - N;
      for (int j = warp; j < T::UH; j += kThreads / 32)
        for (int c = lane; c < T::UP; c += 32) {
          double v = 0.0;
          if (j < R::UH && c < R::UW) {
            const int ux = unk(op.dx, vx0 + c), uy = unk(op.dy, vy0 + j);
            if (ux >= 0 && uy >= 0) v = x[(size_t)uy * op.G0 + ux];
          }
          U[j * T::UP + c] = v;
        }
    }
    for (int k = threadIdx.x; k < T::TW + T::TH; k += kThreads) {
      if (k < T::TW) {
        const int kx = k / N;
        Wx[k] = wsum<N>(op.dx, op.w, ex0 + kx, k - kx * N);
      } else {
        const int r = k - T::TW, ky = r / N;
        Wy[r] = wsum<N>(op.dy, op.w, ey0 + ky, r - ky * N);
      }
    }
    __syncthreads();

    // prefetch the next tile into the other stage (last read one iteration ago)
    const int tn = t + gridDim.x;
    if (threadIdx.x == 0 && tn < ntiles) {
      int xn, yn;
      if (tile_tma<N>(op, tma, tiles_x, tn, xn, yn)) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_expect_tx(&bar[s ^ 1], T::BOX_BYTES);
        tma_load_2d(Ubuf + (s ^ 1) * T::NU, &map, xn & ~1, yn, &bar[s ^ 1]);
      }
    }

    const double* Us = U + off;  // staged (row j, column c) at Us[j * UP + c]

    // rows: units (16-row block rb, element k)
    for (int u = warp; u < T::RB * T::TEX; u += kThreads / 32) {
      const int rb = (u % T::RB) * 16, k = u / T::RB;
      double c[T::NT][4];
#pragma unroll
      for (int nt = 0; nt < T::NT; nt++) c[nt][0] = c[nt][1] = c[nt][2] = c[nt][3] = 0.0;
      const double* w0 = Us + (rb + g + N) * T::UP + k * N;
#pragma unroll
      for (int ks = 0; ks < T::KS; ks++) {
        const double a0 = w0[ks * 8 + tq], a1 = w0[8 * T::UP + ks * 8 + tq];
        const double a2 = w0[ks * 8 + tq + 4], a3 = w0[8 * T::UP + ks * 8 + tq + 4];
#pragma unroll
        for (int nt = 0; nt < T::NT; nt++) dmma(c[nt], a0, a1, a2, a3, bf[ks][nt][0], bf[ks][nt][1]);
      }
#pragma unroll
      for (int nt = 0; nt < T::NT; nt++)
#pragma unroll
        for (int q = 0; q < 4; q++) {
          const int r = rb + g + (q >> 1) * 8, a = nt * 8 + 2 * tq + (q & 1);
          if (r >= T::TH || a >= N) continue;
          const int cc = k * N + a;
          const double uval = Us[(r + N) * T::UP + cc + N];
          double z = c[nt][q];
          if (nat_x && a == 0) {
            const int gx = gx0 + cc;
            if (gx == 0) z = fma(-op.Kh[N * n + N], uval, z);  // no left element
            if (gx == lastx) z = fma(-op.Kh[0], uval, z);      // no own element
          }
          const double wy = Wy[r];
          O[r * T::OP + cc] = fma(op.alpha * Wx[cc] * wy, uval, op.bx * wy * z);
        }
    }
    __syncthreads();

    // columns: units (16-column block cb, element row k); A = window^T
    for (int u = warp; u < T::CB * T::TEY; u += kThreads / 32) {
      const int cb = (u % T::CB) * 16, k = u / T::CB;
      double c[T::NT][4];
#pragma unroll
      for (int nt = 0; nt < T::NT; nt++) c[nt][0] = c[nt][1] = c[nt][2] = c[nt][3] = 0.0;
      const double* w0 = Us + (k * N) * T::UP + cb + g + N;
#pragma unroll
      for (int ks = 0; ks < T::KS; ks++) {
        const double a0 = w0[(ks * 8 + tq) * T::UP], a1 = w0[(ks * 8 + tq) * T::UP + 8];
        const double a2 = w0[(ks * 8 + tq + 4) * T::UP], a3 = w0[(ks * 8 + tq + 4) * T::UP + 8];
#pragma unroll
        for (int nt = 0; nt < T::NT; nt++) dmma(c[nt], a0, a1, a2, a3, bf[ks][nt][0], bf[ks][nt][1]);
      }
#pragma unroll
      for (int nt = 0; nt < T::NT; nt++)
#pragma unroll
        for (int q = 0; q < 4; q++) {
          const int cc = cb + g + (q >> 1) * 8, a = nt * 8 + 2 * tq + (q & 1);
          if (cc >= T::TW || a >= N) continue;
          const int r = k * N + a;
          double z = c[nt][q];
          if (nat_y && a == 0) {
            const int gy = gy0 + r;
            const double uval = Us[(r + N) * T::UP + cc + N];
            if (gy == 0) z = fma(-op.Kh[N * n + N], uval, z);
            if (gy == lasty) z = fma(-op.Kh[0], uval, z);
          }
          const int gx = gx0 + cc, gy = gy0 + r;
          if (gx >= op.dx.lo && gx < op.dx.hi && gy >= op.dy.lo && gy < op.dy.hi)
            y[(size_t)(gy - op.dy.lo) * op.G0 + (gx - op.dx.lo)] =
                fma(op.by * Wx[cc], z, O[r * T::OP + cc]);
        }
    }
    __syncthreads();
  }
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against the driver library).
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

template <int N>
cudaError_t launch_mma(const OpDev& od, const double* x, double* y, unsigned* err, cudaStream_t s) {
  typedef MTile<N> T;
  ApplyOp<double> op;
  for (int k = 0; k < (N + 1) * (N + 1); k++) op.Kh[k] = od.Kh[k];
  for (int k = 0; k <= N; k++) op.w[k] = od.w[k];
  op.alpha = od.alpha;
  op.bx = od.beta[0];
  op.by = od.beta[1];
  op.dx = od.d[0];
  op.dy = od.d[1];
  op.G0 = od.G[0];
  op.G1 = od.G[1];
  static int per_sm[64] = {};  // resident blocks per SM, per instantiation and device
  static int sms[64] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  if (!per_sm[dev]) {
    e = cudaFuncSetAttribute(apply_mma_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)T::SMEM);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&sms[dev], cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    int b = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, apply_mma_kernel<N>, kThreads, T::SMEM);
    if (e != cudaSuccess) return e;
    per_sm[dev] = b > 0 ? b : 1;
  }
  // the tensor map of the unknown array; TMA needs a 16-byte aligned base
  // and a row pitch that is a multiple of 16 bytes
  CUtensorMap map;
  std::memset(&map, 0, sizeof(map));
  int tma = 0;
  PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
  // the TMA path's bounded waits report through err, so it needs one
  if (enc && err && (reinterpret_cast<uintptr_t>(x) & 15) == 0 && (od.G[0] % 2) == 0) {
    const cuuint64_t dims[2] = {(cuuint64_t)od.G[0], (cuuint64_t)od.G[1]};
    const cuuint64_t strides[1] = {(cuuint64_t)od.G[0] * sizeof(double)};
    const cuuint32_t box[2] = {(cuuint32_t)T::UP, (cuuint32_t)T::UH};
    const cuuint32_t estr[2] = {1, 1};
    tma = enc(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<double*>(x), dims, strides, box,
              estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
              CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
  }
  const int tiles_x = (od.d[0].hi + T::TW - 1) / T::TW;
  const int tiles_y = (od.d[1].hi + T::TH - 1) / T::TH;
  const int ntiles = tiles_x * tiles_y;
  const int grid = ntiles < per_sm[dev] * sms[dev] ? ntiles : per_sm[dev] * sms[dev];
  apply_mma_kernel<N><<<grid, kThreads, T::SMEM, s>>>(map, op, x, y, tiles_x, ntiles, tma, err);
  return cudaGetLastError();
}

// ---------------------------------------- orders 4 to 8, CUDA cores ----
// Element-factored FP64 apply on the FP64 FMA pipes for N = 4..8. A block of
// 256 threads stages a TX x TY vertex tile (TX = N * (64 / N): 64, 60, 60,
// 63, 64; TY a multiple of N) and an N-vertex halo to the left and below
// (zero where a vertex is no unknown), then
//   x pass: thread (element e, row r) reads the 2N+1 values of its element
//           row and of the left element's row and forms the N outputs of its
//           element's nodes a = 0..N-1 with the (N+1) x (N+1) stiffness block
//           and, at a = 0, the left element's last row: all coefficients
//           compile-time offsets into the kernel's parameters;
//   y pass: thread (element e, column c) does the same along the column and
//           combines alpha wx wy x + beta_x wy (Kx x) + beta_y wx (Ky x).
// About 2.6 N FMAs and 3 shared-memory loads per unknown, no padding work,
// and the staging costs a few instructions per value (each lane maps its
// staged columns once; a staged row's unknown index is the same for the
// whole warp). The staged row pitch (TX + N + 1, or one more) and the x-pass
// output pitch (TX + 1, or one more) are odd, so a warp's column-wise reads
// are conflict-free.
template <int N>
struct EfTile {
  static constexpr int EX = 64 / N;      // elements per tile row
  static constexpr int TX = EX * N;      // output vertices per tile row
  static constexpr int SW = TX + N + 1;  // staged vertices per row
  static constexpr int W = SW | 1;       // staged row pitch (odd)
  static constexpr int OXP = (TX + 1) | 1;  // x-pass output pitch (odd)
  // output rows per tile: 32, 28, 24, 20, 16 for N = 8, 7, 6, 5, 4
  static constexpr int TY = N == 8 ? 32 : 4 * N;
  static constexpr int H = TY + N + 1;   // staged rows
  static constexpr int ITEMS = EX * TY;  // x-pass (= y-pass) items, one per thread
  static constexpr int MINB = N >= 7 ? 4 : (N == 6 ? 5 : 6);  // blocks per SM
  static_assert(ITEMS <= 256 && TX * (TY / N) == ITEMS && TY % N == 0, "tile shape");
  static_assert(SW <= 96, "staging columns");
};
constexpr int kEfThreads = 256, kEfWarps = kEfThreads / 32;

// Stage the tile's vertices and its N-vertex halo to the left and below into
// X (zero where a vertex is no unknown): warp w takes rows w, w + 8, ...;
// lane l columns l, l + 32, l + 64; all copies issued before the wait.
template <int N, int H = EfTile<N>::H>
__device__ __forceinline__ void ef_stage(const OpDev& op, const double* __restrict__ x, double* X,
                                         int gx0, int gy0) {
  typedef EfTile<N> T;
  constexpr int SW = T::SW, W = T::W;
  const Dir& dx = op.d[0];
  const Dir& dy = op.d[1];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int cu[3];
#pragma unroll
  for (int q = 0; q < 3; q++) {
    const int i = lane + 32 * q;
    cu[q] = i < SW ? unk(dx, gx0 - N + i) : -1;
  }
#pragma unroll
  for (int r = 0; r < (H + kEfWarps - 1) / kEfWarps; r++) {
    const int j = warp + kEfWarps * r;
    if (j < H) {
      const int uy = unk(dy, gy0 - N + j);
      const double* rowp = x + (size_t)(uy < 0 ? 0 : uy) * op.G[0];
#pragma unroll
      for (int q = 0; q < 3; q++) {
        const int i = lane + 32 * q;
        if (i < SW) {
          const bool ok = uy >= 0 && cu[q] >= 0;
          const double* src = ok ? rowp + cu[q] : x;
          const unsigned dst = (unsigned)__cvta_generic_to_shared(X + j * W + i);
          asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(dst), "l"(src),
                       "r"(ok ? 8 : 0));
        }
      }
    }
  }
  asm volatile("cp.async.commit_group;\n" ::);
  asm volatile("cp.async.wait_group 0;\n" ::);
}

template <int N>
__global__ void __launch_bounds__(kEfThreads, EfTile<N>::MINB)
    apply_ef_kernel(const OpDev op, const double* __restrict__ x, double* __restrict__ y) {
  typedef EfTile<N> T;
  constexpr int W = T::W, OXP = T::OXP, TX = T::TX, TY = T::TY, H = T::H;
  extern __shared__ __align__(16) double efsm[];
  double* X = efsm;            // vertices (gx0-N .. gx0+TX) x (gy0-N .. gy0+TY)
  double* OX = X + H * W;      // x-pass results of the tile's vertices
  double* sw = OX + TY * OXP;
  const Dir& dx = op.d[0];
  const Dir& dy = op.d[1];
  const int gx0 = blockIdx.x * TX, gy0 = blockIdx.y * TY;
  const int tid = threadIdx.x;
  if (tid <= N) sw[tid] = op.w[tid];
  ef_stage<N>(op, x, X, gx0, gy0);
  __syncthreads();
  constexpr int n = N + 1;
  if (tid < T::ITEMS) {  // x pass: thread = (element e, row r), rows of one element per warp run
    const int r = tid % TY, e = tid / TY;
    const int ex = gx0 / N + e;
    const double* row = X + (r + N) * W + e * N;  // left element's first node
    double v[2 * N + 1];
#pragma unroll
    for (int k = 0; k <= 2 * N; k++) v[k] = row[k];
    const bool own = ex < dx.nE, left = ex > 0 || dx.periodic;
    double o[N];
#pragma unroll
    for (int a = 0; a < N; a++) {
      double t = 0.0;
      if (own) {
#pragma unroll
        for (int b = 0; b < n; b++) t = fma(op.Kh[a * n + b], v[N + b], t);
      }
      o[a] = t;
    }
    if (left) {
      double t = 0.0;
#pragma unroll
      for (int b = 0; b < n; b++) t = fma(op.Kh[N * n + b], v[b], t);
      o[0] += t;
    }
#pragma unroll
    for (int a = 0; a < N; a++) OX[r * OXP + e * N + a] = o[a];
  }
  __syncthreads();
  if (tid < T::ITEMS) {  // y pass: thread = (element row e, column c), consecutive columns per warp
    const int c = tid % TX, e = tid / TX;
    const int ey = gy0 / N + e;
    const int gx = gx0 + c;
    const double* col = X + (e * N) * W + c + N;  // lower element's first node
    double v[2 * N + 1];
#pragma unroll
    for (int k = 0; k <= 2 * N; k++) v[k] = col[k * W];
    const bool own = ey < dy.nE, left = ey > 0 || dy.periodic;
    double o[N];
#pragma unroll
    for (int a = 0; a < N; a++) {
      double t = 0.0;
      if (own) {
#pragma unroll
        for (int b = 0; b < n; b++) t = fma(op.Kh[a * n + b], v[N + b], t);
      }
      o[a] = t;
    }
    if (left) {
      double t = 0.0;
#pragma unroll
      for (int b = 0; b < n; b++) t = fma(op.Kh[N * n + b], v[b], t);
      o[0] += t;
    }
    if (gx >= dx.lo && gx < dx.hi) {
      const double wx = wsum<N>(dx, sw, gx / N, gx % N);
      const double axw = op.alpha * wx, bxw = op.beta[1] * wx;
      const double w0 = (own ? op.w[0] : 0.0) + (left ? op.w[N] : 0.0);
      const int gyb = gy0 + e * N;
      const size_t ld = (size_t)op.G[0];
      double* yp = y + (ptrdiff_t)(gyb - dy.lo) * op.G[0] + (gx - dx.lo);
      const double* oxp = OX + (e * N) * OXP + c;
      // y = wy (alpha wx x + beta_x (Kx x)) + beta_y wx (Ky x), wy the
      // assembled weight of the row (compile-time parameter offsets)
      if (gyb >= dy.lo && gyb + N <= dy.hi) {  // the whole strip is unknowns
#pragma unroll
        for (int a = 0; a < N; a++) {
          const double wy = a == 0 ? w0 : op.w[a];
          yp[a * ld] = fma(wy, fma(axw, v[N + a], op.beta[0] * oxp[a * OXP]), bxw * o[a]);
        }
      } else {
#pragma unroll
        for (int a = 0; a < N; a++) {
          const int gy = gyb + a;
          const double wy = a == 0 ? w0 : op.w[a];
          const double r = fma(wy, fma(axw, v[N + a], op.beta[0] * oxp[a * OXP]), bxw * o[a]);
          if (gy >= dy.lo && gy < dy.hi) yp[(ptrdiff_t)a * op.G[0]] = r;
        }
      }
    }
  }
}

template <int N>
cudaError_t launch_ef(const OpDev& op, const double* x, double* y, cudaStream_t s) {
  typedef EfTile<N> T;
  constexpr size_t smem = sizeof(double) * ((size_t)T::H * T::W + (size_t)T::TY * T::OXP + 16);
  if (smem > 48 * 1024) {
    static bool attr[64] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (!attr[dev]) {
      e = cudaFuncSetAttribute(apply_ef_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)smem);
      if (e != cudaSuccess) return e;
      attr[dev] = true;
    }
  }
  const dim3 grid((op.d[0].hi + T::TX - 1) / T::TX, (op.d[1].hi + T::TY - 1) / T::TY);
  apply_ef_kernel<N><<<grid, kEfThreads, smem, s>>>(op, x, y);
  return cudaGetLastError();
}

// ------------------------------- refinement residual, orders 4 to 8 ----
// r = b - A x on apply_ef_kernel's tile with TY / kResSplit output rows: the
// stiffness sums of both passes, the combination and the subtraction in
// double-double (the stiffness rows sum to zero, so the taps cancel and a
// plain FP64 sum loses the digits a 1e-10 residual needs), rounded once.
// Each element row (x pass) and column (y pass) is shared by kResSplit
// thread groups, warp-uniform, each forming a contiguous share of its N
// outputs in the same order as one thread would: twice the blocks of half
// the depth for this latency-bound kernel, and the same bits. Per-block
// partial sums of (w r)^2 (or r w r when natural) and r^2; the block that
// finishes last sums the partials in block order and runs the FDM loop's
// convergence test (ResTail). Optionally also writes r's TF32 hi/lo split
// for the tensor-core inverse.
constexpr int kResSplit = 2;
template <int N>
struct ResTile {
  typedef EfTile<N> E;
  static constexpr int EX = E::EX, TX = E::TX, W = E::W, OXP = E::OXP;
  static constexpr int TY = E::TY / kResSplit;   // output rows: 16, 14, 12, 10, 8
  static constexpr int H = TY + N + 1;           // staged rows
  static constexpr int ITEMS = EX * TY;          // rows (x pass) = columns (y pass)
  static constexpr int GROUP = kEfThreads / kResSplit;  // threads of one share
  static constexpr int CH = (N + kResSplit - 1) / kResSplit;  // outputs of a share
  static_assert(TY % N == 0 && ITEMS <= GROUP && GROUP % 32 == 0, "residual tile shape");
};

// x pass of outputs [A0, A1) of one element row: v = the row's 2N+1 staged
// values (left element, shared node, own element).
template <int N, int A0, int A1>
__device__ __forceinline__ void res_xpass(const OpDev& op, const double* row, bool own, bool left,
                                          double* OXH, double* OXL) {
  constexpr int n = N + 1;
  double v[2 * N + 1];
#pragma unroll
  for (int k = (A0 == 0 ? 0 : N); k <= 2 * N; k++) v[k] = row[k];
#pragma unroll
  for (int a = A0; a < A1; a++) {
    double hi = 0.0, lo = 0.0;
    if (own) {
#pragma unroll
      for (int q = 0; q < n; q++) dd_fma(hi, lo, op.Kh[a * n + q], v[N + q]);
    }
    if (A0 == 0 && a == 0 && left) {
      double h2 = 0.0, l2 = 0.0;
#pragma unroll
      for (int q = 0; q < n; q++) dd_fma(h2, l2, op.Kh[N * n + q], v[q]);
      dd_add(hi, lo, h2);
      lo += l2;
    }
    OXH[a] = hi;
    OXL[a] = lo;
  }
}

// y pass, combination and residual of outputs [A0, A1) of one element
// column; accumulates the norm partials.
template <int N, int A0, int A1>
__device__ __forceinline__ void res_ypass(const OpDev& op, const double* col, const double* OXH,
                                          const double* OXL, const double* sw, int c, int e,
                                          int gx, int gy0, bool own, bool left,
                                          const double* __restrict__ b, double* __restrict__ rout,
                                          const double* __restrict__ wv, int natural,
                                          double& acc0, double& acc1, float* __restrict__ sp_hi,
                                          float* __restrict__ sp_lo, int sp_pitch) {
  typedef ResTile<N> T;
  constexpr int n = N + 1, W = T::W, OXP = T::OXP;
  const Dir& dx = op.d[0];
  const Dir& dy = op.d[1];
  double v[2 * N + 1];
#pragma unroll
  for (int k = (A0 == 0 ? 0 : N); k <= 2 * N; k++) v[k] = col[k * W];
  double yh[A1 - A0], yl[A1 - A0];
#pragma unroll
  for (int a = A0; a < A1; a++) {
    double hi = 0.0, lo = 0.0;
    if (own) {
#pragma unroll
      for (int q = 0; q < n; q++) dd_fma(hi, lo, op.Kh[a * n + q], v[N + q]);
    }
    if (A0 == 0 && a == 0 && left) {
      double h2 = 0.0, l2 = 0.0;
#pragma unroll
      for (int q = 0; q < n; q++) dd_fma(h2, l2, op.Kh[N * n + q], v[q]);
      dd_add(hi, lo, h2);
      lo += l2;
    }
    yh[a - A0] = hi;
    yl[a - A0] = lo;
  }
  if (gx < dx.lo || gx >= dx.hi) return;
  const double wx = wsum<N>(dx, sw, gx / N, gx % N);
  const double w0 = (own ? op.w[0] : 0.0) + (left ? op.w[N] : 0.0);
  const int gyb = gy0 + e * N;
  const size_t ux = (size_t)(gx - dx.lo);
#pragma unroll
  for (int a = A0; a < A1; a++) {
    const int gy = gyb + a;
    if (gy < dy.lo || gy >= dy.hi) continue;
    const double wy = a == 0 ? w0 : op.w[a];
    const size_t k = (size_t)(gy - dy.lo) * op.G[0] + ux;
    const double cm = -op.alpha * wx * wy, cx = -op.beta[0] * wy, cy = -op.beta[1] * wx;
    double hi = b[k], lo = 0.0;
    dd_fma(hi, lo, cm, v[N + a]);
    dd_fma(hi, lo, cx, OXH[(e * N + a) * OXP + c]);
    lo = fma(cx, OXL[(e * N + a) * OXP + c], lo);
    dd_fma(hi, lo, cy, yh[a - A0]);
    lo = fma(cy, yl[a - A0], lo);
    const double rv = hi + lo;
    rout[k] = rv;
    const double z = wv ? rv * wv[k] : rv;
    acc0 += natural ? z * rv : z * z;
    acc1 += rv * rv;
    if (sp_hi) {
      uint32_t h;
      asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(h) : "f"((float)rv));
      const float fh = __uint_as_float(h);
      const size_t o = (size_t)(gy - dy.lo) * sp_pitch + ux;
      sp_hi[o] = fh;
      sp_lo[o] = (float)(rv - (double)fh);
    }
  }
}

template <int N>
__global__ void __launch_bounds__(kEfThreads, 2)
    residual_ef_kernel(const OpDev op, const double* __restrict__ x, const double* __restrict__ b,
                       double* __restrict__ rout, const double* __restrict__ wv, int natural,
                       double* __restrict__ partial, const ResTail tail, float* __restrict__ sp_hi,
                       float* __restrict__ sp_lo, int sp_pitch) {
  typedef ResTile<N> T;
  constexpr int W = T::W, OXP = T::OXP, TX = T::TX, TY = T::TY, H = T::H, CH = T::CH;
  extern __shared__ __align__(16) double efsm[];
  double* X = efsm;              // staged vertices
  double* OXH = X + H * W;       // x-pass stiffness sums, high parts
  double* OXL = OXH + TY * OXP;  // and low parts
  double* sw = OXL + TY * OXP;
  __shared__ double red[kEfWarps][2];
  __shared__ unsigned last;
  const Dir& dx = op.d[0];
  const Dir& dy = op.d[1];
  const int gx0 = blockIdx.x * TX, gy0 = blockIdx.y * TY;
  const int tid = threadIdx.x;
  // share of the outputs (warp-uniform) and item of this thread
  const int sub = tid / T::GROUP, item = tid - sub * T::GROUP;
  if (tid <= N) sw[tid] = op.w[tid];
  ef_stage<N, H>(op, x, X, gx0, gy0);
  __syncthreads();
  if (item < T::ITEMS) {  // x pass
    const int r = item % TY, e = item / TY;
    const int ex = gx0 / N + e;
    const double* row = X + (r + N) * W + e * N;
    const bool own = ex < dx.nE, left = ex > 0 || dx.periodic;
    double* oh = OXH + r * OXP + e * N;
    double* ol = OXL + r * OXP + e * N;
    if constexpr (kResSplit == 1)
      res_xpass<N, 0, N>(op, row, own, left, oh, ol);
    else if (sub == 0)
      res_xpass<N, 0, CH>(op, row, own, left, oh, ol);
    else
      res_xpass<N, CH, N>(op, row, own, left, oh, ol);
  }
  __syncthreads();
  double acc0 = 0.0, acc1 = 0.0;
  if (item < T::ITEMS) {  // y pass, the combination and the residual
    const int c = item % TX, e = item / TX;
    const int ey = gy0 / N + e;
    const double* col = X + (e * N) * W + c + N;
    const bool own = ey < dy.nE, left = ey > 0 || dy.periodic;
    if constexpr (kResSplit == 1)
      res_ypass<N, 0, N>(op, col, OXH, OXL, sw, c, e, gx0 + c, gy0, own, left, b, rout, wv,
                         natural, acc0, acc1, sp_hi, sp_lo, sp_pitch);
    else if (sub == 0)
      res_ypass<N, 0, CH>(op, col, OXH, OXL, sw, c, e, gx0 + c, gy0, own, left, b, rout, wv,
                          natural, acc0, acc1, sp_hi, sp_lo, sp_pitch);
    else
      res_ypass<N, CH, N>(op, col, OXH, OXL, sw, c, e, gx0 + c, gy0, own, left, b, rout, wv,
                          natural, acc0, acc1, sp_hi, sp_lo, sp_pitch);
  }
  // block sums in a fixed order
  const int lane = tid & 31, warp = tid >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    acc0 += __shfl_down_sync(0xffffffffu, acc0, o);
    acc1 += __shfl_down_sync(0xffffffffu, acc1, o);
  }
  if (lane == 0) {
    red[warp][0] = acc0;
    red[warp][1] = acc1;
  }
  __syncthreads();
  const unsigned blk = blockIdx.y * gridDim.x + blockIdx.x, nb = gridDim.x * gridDim.y;
  if (tid == 0) {
    double s0 = 0.0, s1 = 0.0;
#pragma unroll
    for (int q = 0; q < kEfWarps; q++) {
      s0 += red[q][0];
      s1 += red[q][1];
    }
    partial[2 * blk] = s0;
    partial[2 * blk + 1] = s1;
  }
  if (!tail.count) return;
  // the last block to finish sums the partials in block order and runs the
  // refinement step's convergence test (no block waits for another)
  __threadfence();
  __syncthreads();
  if (tid == 0) last = atomicAdd(tail.count, 1u) == nb - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  double s0 = 0.0, s1 = 0.0;
  for (unsigned k = tid; k < nb; k += kEfThreads) {
    s0 += __ldcg(partial + 2 * k);
    s1 += __ldcg(partial + 2 * k + 1);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    s0 += __shfl_down_sync(0xffffffffu, s0, o);
    s1 += __shfl_down_sync(0xffffffffu, s1, o);
  }
  __syncthreads();
  if (lane == 0) {
    red[warp][0] = s0;
    red[warp][1] = s1;
  }
  __syncthreads();
  if (tid == 0) {
    double t0 = 0.0, t1 = 0.0;
#pragma unroll
    for (int q = 0; q < kEfWarps; q++) {
      t0 += red[q][0];
      t1 += red[q][1];
    }
    tail.res[0] = t0;
    tail.res[1] = t1;
    *tail.count = 0u;
    fdm_check_state(tail.p, tail.st, t0, tail.h);
  }
}

template <int N>
cudaError_t launch_res_ef(const OpDev& op, const double* x, const double* b, double* r,
                          const double* w, int natural, double* partial, const ResTail& tail,
                          float* sh, float* sl, int sp, cudaStream_t s) {
  typedef ResTile<N> T;
  constexpr size_t smem = sizeof(double) * ((size_t)T::H * T::W + 2 * (size_t)T::TY * T::OXP + 16);
  if (smem > 48 * 1024) {
    static bool attr[64] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (!attr[dev]) {
      e = cudaFuncSetAttribute(residual_ef_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)smem);
      if (e != cudaSuccess) return e;
      attr[dev] = true;
    }
  }
  const dim3 grid((op.d[0].hi + T::TX - 1) / T::TX, (op.d[1].hi + T::TY - 1) / T::TY);
  residual_ef_kernel<N><<<grid, kEfThreads, smem, s>>>(op, x, b, r, w, natural, partial, tail, sh,
                                                       sl, sp);
  return cudaGetLastError();
}

}  // namespace

bool residual_ef_supported(const OpDev& op) {
  return op.gamma == 0.0 && op.d[0].N >= 4 && op.d[0].N <= 8;
}

namespace {
template <int N>
int res_ef_blocks(const OpDev& op) {
  typedef ResTile<N> T;
  return ((op.d[0].hi + T::TX - 1) / T::TX) * ((op.d[1].hi + T::TY - 1) / T::TY);
}
}  // namespace

int residual_partial_blocks(const OpDev& op) {
  if (!residual_ef_supported(op)) return residual_blocks(op);
  switch (op.d[0].N) {
    case 4: return res_ef_blocks<4>(op);
    case 5: return res_ef_blocks<5>(op);
    case 6: return res_ef_blocks<6>(op);
    case 7: return res_ef_blocks<7>(op);
    default: return res_ef_blocks<8>(op);
  }
}

cudaError_t launch_residual_ef(const OpDev& op, const double* x, const double* b, double* r,
                               const double* w, int natural, double* partial, const ResTail& tail,
                               float* split_hi, float* split_lo, int split_pitch, cudaStream_t s) {
  if (!residual_ef_supported(op) || !b || !partial) return cudaErrorInvalidValue;
  switch (op.d[0].N) {
    case 4: return launch_res_ef<4>(op, x, b, r, w, natural, partial, tail, split_hi, split_lo, split_pitch, s);
    case 5: return launch_res_ef<5>(op, x, b, r, w, natural, partial, tail, split_hi, split_lo, split_pitch, s);
    case 6: return launch_res_ef<6>(op, x, b, r, w, natural, partial, tail, split_hi, split_lo, split_pitch, s);
    case 7: return launch_res_ef<7>(op, x, b, r, w, natural, partial, tail, split_hi, split_lo, split_pitch, s);
    default: return launch_res_ef<8>(op, x, b, r, w, natural, partial, tail, split_hi, split_lo, split_pitch, s);
  }
}

#define SE_APPLY_N(n) \
  case n:             \
    return launch_mma<n>(op, x, y, err, s);
cudaError_t launch_op_apply(const OpDev& op, const double* x, double* y, unsigned* err,
                            cudaStream_t s) {
  // an SVV term (dense element blocks) is applied by the CG kernel's staged
  // per-unknown form, which carries it
  if (op.gamma != 0.0) return launch_residual(op, x, nullptr, y, nullptr, 0, nullptr, s);
  switch (op.d[0].N) {
    SE_APPLY_N(2) SE_APPLY_N(3) SE_APPLY_N(9) SE_APPLY_N(10) SE_APPLY_N(11) SE_APPLY_N(12)
    case 4:
      return launch_ef<4>(op, x, y, s);
    case 5:
      return launch_ef<5>(op, x, y, s);
    case 6:
      return launch_ef<6>(op, x, y, s);
    case 7:
      return launch_ef<7>(op, x, y, s);
    case 8:
      return launch_ef<8>(op, x, y, s);
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
  if (op.gamma != 0.0) return cudaErrorNotSupported;  // no SVV term in the low-precision apply
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
