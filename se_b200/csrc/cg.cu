// Persistent, deterministic Jacobi-preconditioned CG over a batch of
// Helmholtz/Poisson solves of one polynomial order N, sm_100a.
//
// One cooperative launch runs every iteration of every solve in the batch.
// The unknown grid of each solve is cut into tiles of kCgTileX x kCgTileY
// unknowns, assigned in contiguous chunks to the resident blocks, one
// unknown per thread and tile.
//
//  * Resident mode (K > 0, each block owns at most K tiles): x, r, the
//    Jacobi inverse, p and A p of a thread's unknowns stay in registers for
//    the whole solve. Only z and p go to memory each iteration, because the
//    neighbouring tiles read them as their stencil halo.
//  * Streaming mode (K == 0, any size): the same iteration with x, r, w and
//    the Jacobi inverse in memory; bounded by HBM bandwidth.
//
// The operator is the tensor-product form of SE's assembled c*Mass +
// s*Laplacian (see linsys.cu); each tile is staged with its halo in shared
// memory and every unknown sums its row of the assembled 1-D operators in a
// fixed order, so there are no atomics and results are bit-for-bit
// repeatable.
//
// Dot products: every block accumulates per-segment partial sums (a
// segment is a run of one solve's tiles inside one block) and, after each
// grid barrier, every block sums every solve's segments in the same fixed
// order; all blocks therefore hold identical scalars and take identical
// decisions without another round trip. The iteration and its tests are
// PETSc's KSPCG with PCJACOBI as SE runs it (src/linsys/HelmholtzEqn.cpp:
// 141-150): zero initial guess, preconditioned/unpreconditioned/natural
// norm, RTOL/ATOL/DTOL/ITS, and the sign checks for an indefinite matrix
// or preconditioner; a constant null space is projected out of every
// preconditioned residual. With remove_null == 2 the right-hand side b is
// first replaced by b - (sum b / sum d) d (d the operator diagonal): the
// system whose solution that iteration approaches. On a b already in the
// operator's range this changes nothing beyond rounding; on a b off it (a
// divergence formed at the vertices, say) PETSc's iteration (remove_null ==
// 1) stagnates at the size of the off-range part and ends on an indefinite
// inner product, where this one converges.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "common.cuh"
#include "fdm_ctl.cuh"

namespace seg {
namespace {

struct SolveState {
  double beta, betaold, dpi, bcoef, a, rnorm0, ttol, dp, zmean, cproj;
  int its, done, reason, pbuf;
};
struct SolveMeta {
  int seg_begin, seg_end, max_it, norm_type, remove_null, n;
  double rtol, atol, dtol;
};

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Grid barrier for a cooperative launch: block 0 adds 2^31 - (nblocks - 1),
// every other block adds 1, so the word's top bit flips exactly when all
// blocks have arrived; no reset is needed between uses. The wait is bounded:
// after 2^26 polls a block records KERR_BARRIER_TIMEOUT and returns false.
constexpr long kPollLimit = 1L << 26;
__device__ __forceinline__ bool grid_sync(unsigned* bar, unsigned* err) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned inc = blockIdx.x == 0 ? 0x80000000u - (gridDim.x - 1u) : 1u;
    __threadfence();
    const unsigned old = atomicAdd(bar, inc);
    long polls = 0;
    int ok = 1;
    while (((ld_acquire_u32(bar) ^ old) & 0x80000000u) == 0u) {
      if (++polls > kPollLimit) {
        atomicOr(err, KERR_BARRIER_TIMEOUT);
        ok = 0;
        break;
      }
    }
    __threadfence();
    s_ok = ok;
  }
  __syncthreads();
  return s_ok;
}

// Fixed-order block reduction of 4 sums; the result is valid in thread 0.
__device__ __forceinline__ void block_sum4(double v[4], double (*sm)[4]) {
#pragma unroll
  for (int q = 0; q < 4; q++)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0)
#pragma unroll
    for (int q = 0; q < 4; q++) sm[w][q] = v[q];
  __syncthreads();
  if (w == 0) {
#pragma unroll
    for (int q = 0; q < 4; q++) {
      v[q] = l < kCgThreads / 32 ? sm[l][q] : 0.0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_down_sync(0xffffffffu, v[q], o);
    }
  }
  __syncthreads();
}

// All four partial slots of one solve's segments at once (one 32-byte load
// per segment), fixed order; every lane of the calling warp gets the sums.
__device__ __forceinline__ void seg_sum4(const double* partials, int b, int e, double out[4]) {
  const int l = threadIdx.x & 31;
  double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
  for (int k = b + l; k < e; k += 32) {
    const double2* p = reinterpret_cast<const double2*>(partials + (size_t)k * 4);
    const double2 u = p[0], v = p[1];
    s0 += u.x;
    s1 += u.y;
    s2 += v.x;
    s3 += v.y;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    s0 += __shfl_xor_sync(0xffffffffu, s0, o);
    s1 += __shfl_xor_sync(0xffffffffu, s1, o);
    s2 += __shfl_xor_sync(0xffffffffu, s2, o);
    s3 += __shfl_xor_sync(0xffffffffu, s3, o);
  }
  out[0] = s0;
  out[1] = s1;
  out[2] = s2;
  out[3] = s3;
}

// ---------------------------------------------------------------- operator --
template <int N>
struct Geo {
  static constexpr int W = kCgTileX + 2 * N;
  static constexpr int H = kCgTileY + 2 * N;
  static constexpr int kRows = kCgTileY * W;       // tile rows, full width
  static constexpr int kCols = 2 * N * kCgTileX;   // tile columns, y-halo only
  static constexpr int kCorners = 4 * N * N;       // the halo's corners
};

// Unknown index of unwrapped vertex g along d (-1: Dirichlet or outside).
__device__ __forceinline__ int unknown_1d(const Dir& d, int g) {
  if (d.periodic) {
    const int L = d.nV - 1;
    if (g < 0) g += L;
    else if (g >= L) g -= L;
  } else if (g < 0 || g >= d.nV) {
    return -1;
  }
  return (g >= d.lo && g < d.hi) ? g - d.lo : -1;
}

// Assembled 1-D GLL weight and stiffness diagonal at vertex g (e = g/N, a).
template <int N, class T = double>
__device__ __forceinline__ T wsum_n(const Dir& d, const T* w, int e, int a) {
  T s = T(0);
  if (e < d.nE) s += w[a];
  if (a == 0 && (e > 0 || d.periodic)) s += w[N];
  return s;
}
template <int N>
__device__ __forceinline__ double kdiag_n(const Dir& d, const double* Kh, int e, int a) {
  constexpr int n = N + 1;
  double s = 0.0;
  if (e < d.nE) s += Kh[a * n + a];
  if (a == 0 && (e > 0 || d.periodic)) s += Kh[N * n + N];
  return s;
}
// Row of the assembled 1-D stiffness at vertex (e, a) applied to the staged
// values around c (stride between neighbouring vertices).
template <int N, int STRIDE, class T = double>
__device__ __forceinline__ T krow_n(const Dir& d, const T* Kh, int e, int a, const T* c) {
  constexpr int n = N + 1;
  T s = T(0);
  if (a != 0) {
    const T* k = Kh + a * n;
    const T* q = c - a * STRIDE;
#pragma unroll
    for (int b = 0; b < n; b++) s = fma(k[b], q[b * STRIDE], s);
    return s;
  }
  if (e > 0 || d.periodic) {
    const T* k = Kh + N * n;
#pragma unroll
    for (int b = 0; b < n; b++) s = fma(k[b], c[(b - N) * STRIDE], s);
  }
  if (e < d.nE) {
#pragma unroll
    for (int b = 0; b < n; b++) s = fma(Kh[b], c[b * STRIDE], s);
  }
  return s;
}

// Per-block copy of one solve's operator coefficients.
struct OpSm {
  double Kh[SE_MAXN1 * SE_MAXN1];
  double Sv[SE_MAXN1 * SE_MAXN1], Tv[SE_MAXN1 * SE_MAXN1];  // SVV factors (gamma != 0)
  double w[SE_MAXN1];
  double alpha, beta0, beta1, gamma;
  // FP32 copies for the reduced-precision apply
  float Khf[SE_MAXN1 * SE_MAXN1], wf[SE_MAXN1];
  float alphaf, beta0f, beta1f;
  Dir dx, dy;
  int G0, G1;
  int solve;
  const double* b;
  double *x, *r, *z, *p0, *p1, *wv, *dinv;
};

__device__ __forceinline__ void load_op(OpSm& o, const CgSolve& S, int solve) {
  if (o.solve == solve) return;
  __syncthreads();
  const OpDev& op = S.op;
  const int n = op.d[0].N + 1;
  for (int k = threadIdx.x; k < n * n; k += blockDim.x) {
    o.Kh[k] = op.Kh[k];
    o.Khf[k] = (float)op.Kh[k];
  }
  if (op.gamma != 0.0)
    for (int k = threadIdx.x; k < n * n; k += blockDim.x) {
      o.Sv[k] = op.Sv[k];
      o.Tv[k] = op.Tv[k];
    }
  if (threadIdx.x < n) {
    o.w[threadIdx.x] = op.w[threadIdx.x];
    o.wf[threadIdx.x] = (float)op.w[threadIdx.x];
  }
  if (threadIdx.x == 0) {
    o.alpha = op.alpha;
    o.beta0 = op.beta[0];
    o.beta1 = op.beta[1];
    o.alphaf = (float)op.alpha;
    o.beta0f = (float)op.beta[0];
    o.beta1f = (float)op.beta[1];
    o.gamma = op.gamma;
    o.dx = op.d[0];
    o.dy = op.d[1];
    o.G0 = op.G[0];
    o.G1 = op.G[1];
    o.solve = solve;
    o.b = S.b;
    o.x = S.x;
    o.r = S.r;
    o.z = S.z;
    o.p0 = S.p0;
    o.p1 = S.p1;
    o.wv = S.w;
    o.dinv = S.dinv;
  }
  __syncthreads();
}

// Stage p = z + bc*p_old (p = z when first) for the tile and its halo: the
// cross the Kronecker-sum terms read (the tile's rows at full width, its
// columns at full height), and with an SVV term also the four N x N corners,
// which its element blocks reach.
// The value a staged p takes: FP64 (LP 0), or rounded to BF16 (LP 1) or
// FP16 (LP 2) and held as FP32, the reduced-precision apply's input.
template <int LP>
__device__ __forceinline__ auto lp_value(double v) {
  if constexpr (LP == 0)
    return v;
  else if constexpr (LP == 1)
    return __bfloat162float(__double2bfloat16(v));
  else
    return __half2float(__double2half(v));
}

template <int N, int LP = 0>
__device__ __forceinline__ void stage_p(const OpSm& o, int x0, int y0, const double* z,
                                        const double* po, bool first, double bc,
                                        decltype(lp_value<LP>(0.0))* P) {
  typedef Geo<N> G;
  const int gx0 = x0 + o.dx.lo - N, gy0 = y0 + o.dy.lo - N;
  const int total = G::kRows + G::kCols + (o.gamma != 0.0 ? G::kCorners : 0);
  // A tile whose staged window lies inside the unknown range of both
  // directions (no periodic wrap, no Dirichlet or outside vertex) indexes its
  // unknowns affinely; the others map each vertex (unknown_1d).
  const bool interior = gx0 >= o.dx.lo && gx0 + G::W <= o.dx.hi && gy0 >= o.dy.lo &&
                        gy0 + G::H <= o.dy.hi;
  const size_t base = interior ? (size_t)(gy0 - o.dy.lo) * o.G0 + (gx0 - o.dx.lo) : 0;
  // every load of the thread issued before any is used (one memory round
  // trip per tile instead of one per staged value)
  constexpr int MAXK = (G::kRows + G::kCols + G::kCorners + kCgThreads - 1) / kCgThreads;
  double v[MAXK];
  int pos[MAXK];
#pragma unroll
  for (int t = 0; t < MAXK; t++) {
    const int k = threadIdx.x + t * kCgThreads;
    v[t] = 0.0;
    pos[t] = -1;
    if (k >= total) continue;
    int i, j;
    if (k < G::kRows) {
      j = N + k / G::W;
      i = k - (j - N) * G::W;
    } else if (k < G::kRows + G::kCols) {
      const int q = k - G::kRows;
      const int jj = q / kCgTileX;
      i = N + (q - jj * kCgTileX);
      j = jj < N ? jj : jj + kCgTileY;
    } else {
      const int q = k - G::kRows - G::kCols;
      const int cj = q / (2 * N), ci = q - cj * (2 * N);
      i = ci < N ? ci : ci + kCgTileX;
      j = cj < N ? cj : cj + kCgTileY;
    }
    pos[t] = j * G::W + i;
    long q = -1;
    if (interior) {
      q = (long)(base + (size_t)j * o.G0 + i);
    } else {
      const int ux = unknown_1d(o.dx, gx0 + i), uy = unknown_1d(o.dy, gy0 + j);
      if (ux >= 0 && uy >= 0) q = (long)uy * o.G0 + ux;
    }
    if (q >= 0) v[t] = first ? z[q] : fma(bc, po[q], z[q]);
  }
#pragma unroll
  for (int t = 0; t < MAXK; t++)
    if (pos[t] >= 0) P[pos[t]] = lp_value<LP>(v[t]);
  __syncthreads();
}

// SVV term (Sv along x (x) Tv along y) at the unknown staged at c (vertex
// (ex, ax), (ey, ay)): over the up to four elements holding the vertex, the
// vertex's row of each element block applied to that element's staged
// values, x contraction first.
template <int N>
__device__ __forceinline__ double svv_n(const OpSm& o, const double* c, int ex, int ax, int ey,
                                        int ay) {
  typedef Geo<N> G;
  constexpr int n = N + 1;
  auto elem = [&](int lx, int ly) {
    const double* srow = o.Sv + lx * n;
    const double* trow = o.Tv + ly * n;
    const double* q = c - ly * G::W - lx;
    double t = 0.0;
#pragma unroll
    for (int b = 0; b < n; b++) {
      double r = 0.0;
#pragma unroll
      for (int a = 0; a < n; a++) r = fma(srow[a], q[b * G::W + a], r);
      t = fma(trow[b], r, t);
    }
    return t;
  };
  // the element to the right/above (local index ax, ay) exists unless the
  // vertex ends a non-periodic mesh; the one to the left/below (local index
  // N) when the vertex starts an element other than a non-periodic first
  const bool xr = ax != 0 || ex < o.dx.nE, xl = ax == 0 && (ex > 0 || o.dx.periodic);
  const bool yr = ay != 0 || ey < o.dy.nE, yl = ay == 0 && (ey > 0 || o.dy.periodic);
  double s = 0.0;
  if (xr && yr) s += elem(ax, ay);
  if (xl && yr) s += elem(N, ay);
  if (xr && yl) s += elem(ax, N);
  if (xl && yl) s += elem(N, N);
  return s;
}

// (A p) at the thread's unknown (tile coordinates tx, ty; vertex gx, gy).
template <int N>
__device__ __forceinline__ double apply_n(const OpSm& o, const double* P, int tx, int ty, int gx,
                                          int gy) {
  typedef Geo<N> G;
  const double* c = P + (ty + N) * G::W + (tx + N);
  const int ex = gx / N, ax = gx - ex * N, ey = gy / N, ay = gy - ey * N;
  const double wx = wsum_n<N>(o.dx, o.w, ex, ax), wy = wsum_n<N>(o.dy, o.w, ey, ay);
  const double kx = krow_n<N, 1>(o.dx, o.Kh, ex, ax, c);
  const double ky = krow_n<N, G::W>(o.dy, o.Kh, ey, ay, c);
  const double a = o.alpha * wx * wy * c[0] + o.beta0 * wy * kx + o.beta1 * wx * ky;
  return o.gamma != 0.0 ? a + o.gamma * svv_n<N>(o, c, ex, ax, ey, ay) : a;
}

// (A p) in FP32 arithmetic on the staged reduced-precision p (no SVV term):
// the same sums as apply_n, FP32 coefficients and accumulation.
template <int N>
__device__ __forceinline__ float apply_lp(const OpSm& o, const float* P, int tx, int ty, int gx,
                                          int gy) {
  typedef Geo<N> G;
  const float* c = P + (ty + N) * G::W + (tx + N);
  const int ex = gx / N, ax = gx - ex * N, ey = gy / N, ay = gy - ey * N;
  const float wx = wsum_n<N, float>(o.dx, o.wf, ex, ax), wy = wsum_n<N, float>(o.dy, o.wf, ey, ay);
  const float kx = krow_n<N, 1, float>(o.dx, o.Khf, ex, ax, c);
  const float ky = krow_n<N, G::W, float>(o.dy, o.Khf, ey, ay, c);
  return o.alphaf * wx * wy * c[0] + o.beta0f * wy * kx + o.beta1f * wx * ky;
}

template <int N>
__device__ __forceinline__ double diag_n(const OpSm& o, int gx, int gy) {
  const int ex = gx / N, ax = gx - ex * N, ey = gy / N, ay = gy - ey * N;
  const double wx = wsum_n<N>(o.dx, o.w, ex, ax), wy = wsum_n<N>(o.dy, o.w, ey, ay);
  const double d = o.alpha * wx * wy + o.beta0 * kdiag_n<N>(o.dx, o.Kh, ex, ax) * wy +
                   o.beta1 * wx * kdiag_n<N>(o.dy, o.Kh, ey, ay);
  if (o.gamma == 0.0) return d;
  return d + o.gamma * kdiag_n<N>(o.dx, o.Sv, ex, ax) * kdiag_n<N>(o.dy, o.Tv, ey, ay);
}

// --------------------------------------------------------------- scalars --
// KSPConvergedDefault on the residual norm dp at iteration n.
__device__ __forceinline__ void converged(SolveState& s, const SolveMeta& m, int n, double dp) {
  if (!(dp == dp) || isinf(dp)) {
    s.reason = -9;
    s.done = 1;
    return;
  }
  if (n == 0) {
    s.rnorm0 = dp;
    s.ttol = fmax(m.rtol * dp, m.atol);
  }
  if (dp <= s.ttol) {
    s.reason = dp < m.atol ? 3 : 2;
    s.done = 1;
  } else if (n > 0 && dp >= m.dtol * s.rnorm0) {
    s.reason = -4;
    s.done = 1;
  }
}
__device__ __forceinline__ double norm_of(const SolveMeta& m, double zz, double zr, double rr) {
  return m.norm_type == 0 ? sqrt(zz) : (m.norm_type == 1 ? sqrt(rr) : sqrt(fabs(zr)));
}

enum Step { ST_PROJ = 0, ST_MEAN, ST_START, ST_APPLY, ST_UPDATE };

// After a barrier: every block updates every solve's state from the partial
// sums, warp w taking solves w, w + nwarps, ...; then counts active solves.
template <int STEP>
__device__ __forceinline__ int update_states(const CgBatch& B, const double* part, SolveState* st,
                                             const SolveMeta* mt) {
  __shared__ int s_active;
  if (threadIdx.x == 0) s_active = 0;
  __syncthreads();
  const int w = threadIdx.x >> 5, nw = kCgThreads / 32, l = threadIdx.x & 31;
  for (int s = w; s < B.nsolves; s += nw) {
    SolveState& S = st[s];
    const SolveMeta& M = mt[s];
    if (STEP != ST_MEAN && STEP != ST_PROJ && S.done) continue;
    double v[4];
    seg_sum4(part, M.seg_begin, M.seg_end, v);
    if (l != 0) continue;
    if (STEP == ST_PROJ) {
      S.cproj = M.remove_null == 2 ? v[0] / v[1] : 0.0;
    } else if (STEP == ST_MEAN) {
      S.zmean = M.remove_null ? v[3] / M.n : 0.0;
    } else if (STEP == ST_START) {
      const double dp = norm_of(M, v[0], v[1], v[2]);
      S.dp = dp;
      converged(S, M, 0, dp);
      S.beta = v[1];
      if (!S.done && M.max_it <= 0) {
        S.reason = -3;
        S.done = 1;
      }
      if (!S.done && S.beta == 0.0) {
        S.reason = 3;
        S.done = 1;
      }
    } else if (STEP == ST_APPLY) {
      const double dpi = v[0];
      const double dpiold = S.dpi;
      S.dpi = dpi;
      S.betaold = S.beta;
      S.pbuf ^= 1;
      if (dpi == 0.0 || (S.its > 0 && dpi * dpiold <= 0.0)) {
        S.reason = -10;
        S.done = 1;
      } else {
        S.a = S.beta / dpi;
      }
    } else {
      const double zr = v[1];
      S.its += 1;
      const double dp = norm_of(M, v[0], v[1], v[2]);
      S.dp = dp;
      converged(S, M, S.its, dp);
      if (!S.done) {
        if (zr == 0.0) {
          S.reason = 3;
          S.done = 1;
        } else if (zr * S.betaold < 0.0) {
          S.reason = -8;
          S.done = 1;
        } else if (S.its >= M.max_it) {
          S.reason = -3;
          S.done = 1;
        } else {
          S.beta = zr;
          S.bcoef = zr / S.betaold;
        }
      }
    }
  }
  __syncthreads();
  for (int s = threadIdx.x; s < B.nsolves; s += kCgThreads)
    if (!st[s].done) atomicAdd(&s_active, 1);
  __syncthreads();
  return s_active;
}

enum Pass { PS_PROJ = 0, PS_INIT, PS_NULL, PS_APPLY, PS_UPDATE };

template <int N, int K>
struct Regs {
  double x[K > 0 ? K : 1], r[K > 0 ? K : 1], dinv[K > 0 ? K : 1], p[K > 0 ? K : 1],
      w[K > 0 ? K : 1], z[K > 0 ? K : 1];
};

// One pass over the block's tiles; writes the block's segment partials.
constexpr int kTileCache = 64;  // tile descriptors a block keeps in shared memory

template <int N, int K, int PASS, int LP = 0>
__device__ __forceinline__ void pass(const CgBatch& B, double* part, const SolveState* st, OpSm& o,
                                     double* P, double (*red)[4], Regs<N, K>& R, int t0, int t1,
                                     const CgTile* tcache) {
  const int tx = threadIdx.x & (kCgTileX - 1), ty = threadIdx.x / kCgTileX;
  int seg = -1;
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  // The tile loop body; `continue` in it means "next tile".
  auto tile = [&](int kk, int t) {
    const CgTile T = t - t0 < kTileCache ? tcache[t - t0] : B.tiles[t];
    if (T.seg != seg) {
      if (seg >= 0) {
        block_sum4(acc, red);
        if (threadIdx.x == 0)
#pragma unroll
          for (int q = 0; q < 4; q++) part[(size_t)seg * 4 + q] = acc[q];
      }
      seg = T.seg;
#pragma unroll
      for (int q = 0; q < 4; q++) acc[q] = 0.0;
    }
    const SolveState& S = st[T.solve];
    if (S.done && PASS != PS_INIT && PASS != PS_PROJ) return;
    load_op(o, B.solves[T.solve], T.solve);
    const int ux = T.x0 + tx, uy = T.y0 + ty;
    const bool in = ux < o.G0 && uy < o.G1;
    const size_t k = (size_t)uy * o.G0 + ux;
    const int gx = ux + o.dx.lo, gy = uy + o.dy.lo;
    if (PASS == PS_APPLY) {
      const double* po = S.pbuf ? o.p1 : o.p0;
      double* pn = S.pbuf ? o.p0 : o.p1;
      double p = 0.0, w = 0.0;
      if constexpr (LP == 0) {
        stage_p<N>(o, T.x0, T.y0, o.z, po, S.its == 0, S.bcoef, P);
        if (in) {
          p = P[(ty + N) * Geo<N>::W + (tx + N)];
          w = apply_n<N>(o, P, tx, ty, gx, gy);
        }
      } else {
        float* PF = reinterpret_cast<float*>(P);
        stage_p<N, LP>(o, T.x0, T.y0, o.z, po, S.its == 0, S.bcoef, PF);
        if (in) {
          p = S.its == 0 ? o.z[k] : fma(S.bcoef, po[k], o.z[k]);  // the FP64 direction
          w = (double)apply_lp<N>(o, PF, tx, ty, gx, gy);
        }
      }
      if (in) {
        pn[k] = p;
        if (K > 0) {
          R.p[kk] = p;
          R.w[kk] = w;
        } else {
          o.wv[k] = w;
        }
        acc[0] += p * w;
      }
      __syncthreads();  // the next tile reuses P
      return;
    }
    if (!in) return;
    if (PASS == PS_PROJ) {  // sums of b and of the diagonal
      acc[0] += o.b[k];
      acc[1] += diag_n<N>(o, gx, gy);
    } else if (PASS == PS_INIT) {
      const double d = diag_n<N>(o, gx, gy);
      const double r = o.b[k] - S.cproj * d;
      const double di = 1.0 / d;
      const double z = r * di;
      if (K > 0) {
        R.x[kk] = 0.0;
        R.r[kk] = r;
        R.dinv[kk] = di;
        R.z[kk] = z;
      } else {
        o.x[k] = 0.0;
        o.r[k] = r;
        o.dinv[k] = di;
      }
      o.z[k] = z;
      acc[0] += z * z;
      acc[1] += z * r;
      acc[2] += r * r;
      acc[3] += z;
    } else if (PASS == PS_NULL) {
      const double z = (K > 0 ? R.z[kk] : o.z[k]) - S.zmean;
      const double r = K > 0 ? R.r[kk] : o.r[k];
      if (K > 0) R.z[kk] = z;
      o.z[k] = z;
      acc[0] += z * z;
      acc[1] += z * r;
      acc[2] += r * r;
    } else {  // PS_UPDATE: x += a p; r -= a w; z = D^-1 r
      const double a = S.a;
      double x, r, di;
      if (K > 0) {
        x = fma(a, R.p[kk], R.x[kk]);
        r = fma(-a, R.w[kk], R.r[kk]);
        di = R.dinv[kk];
        R.x[kk] = x;
        R.r[kk] = r;
      } else {
        const double* pc = S.pbuf ? o.p1 : o.p0;  // pbuf already points at the new p
        x = fma(a, pc[k], o.x[k]);
        r = fma(-a, o.wv[k], o.r[k]);
        di = o.dinv[k];
        o.x[k] = x;
        o.r[k] = r;
      }
      const double z = r * di;
      if (K > 0) R.z[kk] = z;
      o.z[k] = z;
      acc[0] += z * z;
      acc[1] += z * r;
      acc[2] += r * r;
      acc[3] += z;
    }
    };
  if (K > 0) {
#pragma unroll
    for (int kk = 0; kk < (K > 0 ? K : 1); kk++)
      if (t0 + kk < t1) tile(kk, t0 + kk);
  } else {
    for (int t = t0; t < t1; t++) tile(0, t);
  }
  if (seg >= 0) {
    block_sum4(acc, red);
    if (threadIdx.x == 0)
#pragma unroll
      for (int q = 0; q < 4; q++) part[(size_t)seg * 4 + q] = acc[q];
  }
}

template <int N, int K, int LP = 0>
__global__ void __launch_bounds__(kCgThreads, 1) cg_n_kernel(const CgBatch B) {
  extern __shared__ double dyn[];
  SolveState* st = reinterpret_cast<SolveState*>(dyn);
  SolveMeta* mt = reinterpret_cast<SolveMeta*>(st + B.nsolves);
  double* P = reinterpret_cast<double*>(mt + B.nsolves);
  P = reinterpret_cast<double*>((reinterpret_cast<uintptr_t>(P) + 15) & ~uintptr_t(15));
  __shared__ OpSm o;
  __shared__ double red[kCgThreads / 32][4];
  __shared__ CgTile tcache[kTileCache];
  Regs<N, K> R;
  const int t0 = B.block_tile_begin[blockIdx.x], t1 = B.block_tile_begin[blockIdx.x + 1];
  if (threadIdx.x == 0) o.solve = -1;
  for (int t = t0 + threadIdx.x; t < t1 && t - t0 < kTileCache; t += kCgThreads)
    tcache[t - t0] = B.tiles[t];
  bool any_null = false, any_proj = false;
  for (int s = threadIdx.x; s < B.nsolves; s += kCgThreads) {
    const CgSolve& C = B.solves[s];
    SolveMeta& M = mt[s];
    M.seg_begin = C.seg_begin;
    M.seg_end = C.seg_end;
    M.max_it = C.max_it;
    M.norm_type = C.norm_type;
    M.remove_null = C.remove_null;
    M.n = C.n;
    M.rtol = C.rtol;
    M.atol = C.atol;
    M.dtol = C.dtol;
    SolveState& S = st[s];
    S.beta = S.betaold = S.dpi = S.bcoef = S.a = S.rnorm0 = S.ttol = S.dp = S.zmean = S.cproj =
        0.0;
    S.its = S.done = S.reason = S.pbuf = 0;
  }
  __syncthreads();
  for (int s = 0; s < B.nsolves; s++) {
    any_null |= mt[s].remove_null != 0;
    any_proj |= mt[s].remove_null == 2;
  }

  // Partial sums alternate between two buffers pass by pass: a block that
  // has passed barrier k may write pass k+1's sums while a slower block still
  // reads pass k's, but nobody writes pass k+2's before every block has
  // arrived at barrier k+1, i.e. finished reading pass k's.
  int pc = 0;
  auto part = [&]() { return B.partials + (size_t)(pc & 1) * B.nseg * 4; };
  if (any_proj) {
    pass<N, K, PS_PROJ>(B, part(), st, o, P, red, R, t0, t1, tcache);
    if (!grid_sync(B.bar_count, B.err)) return;
    update_states<ST_PROJ>(B, part(), st, mt);
    ++pc;
  }
  pass<N, K, PS_INIT>(B, part(), st, o, P, red, R, t0, t1, tcache);
  if (!grid_sync(B.bar_count, B.err)) return;
  update_states<ST_MEAN>(B, part(), st, mt);
  if (any_null) {
    ++pc;
    pass<N, K, PS_NULL>(B, part(), st, o, P, red, R, t0, t1, tcache);
    if (!grid_sync(B.bar_count, B.err)) return;
  }
  int active = update_states<ST_START>(B, part(), st, mt);
  while (active > 0) {
    ++pc;
    pass<N, K, PS_APPLY, LP>(B, part(), st, o, P, red, R, t0, t1, tcache);
    if (!grid_sync(B.bar_count, B.err)) return;
    update_states<ST_APPLY>(B, part(), st, mt);
    ++pc;
    pass<N, K, PS_UPDATE>(B, part(), st, o, P, red, R, t0, t1, tcache);
    if (!grid_sync(B.bar_count, B.err)) return;
    if (any_null) {
      update_states<ST_MEAN>(B, part(), st, mt);
      ++pc;
      pass<N, K, PS_NULL>(B, part(), st, o, P, red, R, t0, t1, tcache);
      if (!grid_sync(B.bar_count, B.err)) return;
    }
    active = update_states<ST_UPDATE>(B, part(), st, mt);
  }
  // results: x back to memory (resident mode), states by block 0
  if (K > 0) {
    const int tx = threadIdx.x & (kCgTileX - 1), ty = threadIdx.x / kCgTileX;
#pragma unroll
    for (int kk = 0; kk < (K > 0 ? K : 1); kk++) {
      const int t = t0 + kk;
      if (t >= t1) break;
      const CgTile T = B.tiles[t];
      const CgSolve& C = B.solves[T.solve];
      const int ux = T.x0 + tx, uy = T.y0 + ty;
      if (ux < C.op.G[0] && uy < C.op.G[1]) C.x[(size_t)uy * C.op.G[0] + ux] = R.x[kk];
    }
  }
  if (blockIdx.x == 0)
    for (int s = threadIdx.x; s < B.nsolves; s += kCgThreads) {
      CgSolve& C = B.solves[s];
      const SolveState& S = st[s];
      C.its = S.its;
      C.reason = S.reason;
      C.done = S.done;
      C.dp = S.dp;
      C.rnorm0 = S.rnorm0;
      C.beta = S.beta;
    }
}



// ------------------------------------------- extended-precision residual --
// krow_n in double-double: the stiffness rows sum to zero, so the taps cancel
// and a plain FP64 sum loses the digits a 1e-10 residual needs.
template <int N, int STRIDE>
__device__ __forceinline__ void krow_dd(const Dir& d, const double* Kh, int e, int a, const double* c,
                                        double& hi, double& lo) {
  constexpr int n = N + 1;
  hi = 0.0;
  lo = 0.0;
  if (a != 0) {
    const double* k = Kh + a * n;
    const double* q = c - a * STRIDE;
#pragma unroll
    for (int b = 0; b < n; b++) dd_fma(hi, lo, k[b], q[b * STRIDE]);
    return;
  }
  if (e > 0 || d.periodic) {
    const double* k = Kh + N * n;
#pragma unroll
    for (int b = 0; b < n; b++) dd_fma(hi, lo, k[b], c[(b - N) * STRIDE]);
  }
  if (e < d.nE) {
#pragma unroll
    for (int b = 0; b < n; b++) dd_fma(hi, lo, Kh[b], c[b * STRIDE]);
  }
}
// b - (A p) at the thread's unknown, accumulated in double-double and
// rounded once.
template <int N>
__device__ __forceinline__ double residual_dd(const OpSm& o, const double* P, int tx, int ty, int gx,
                                              int gy, double bval) {
  typedef Geo<N> G;
  const double* c = P + (ty + N) * G::W + (tx + N);
  const int ex = gx / N, ax = gx - ex * N, ey = gy / N, ay = gy - ey * N;
  const double wx = wsum_n<N>(o.dx, o.w, ex, ax), wy = wsum_n<N>(o.dy, o.w, ey, ay);
  double kxh, kxl, kyh, kyl;
  krow_dd<N, 1>(o.dx, o.Kh, ex, ax, c, kxh, kxl);
  krow_dd<N, G::W>(o.dy, o.Kh, ey, ay, c, kyh, kyl);
  double hi = bval, lo = 0.0;
  const double cm = -o.alpha * wx * wy, cx = -o.beta0 * wy, cy = -o.beta1 * wx;
  dd_fma(hi, lo, cm, c[0]);
  dd_fma(hi, lo, cx, kxh);
  lo = fma(cx, kxl, lo);
  dd_fma(hi, lo, cy, kyh);
  lo = fma(cy, kyl, lo);
  return hi + lo;
}

// ------------------------------------------- standalone apply / residual --
// y = A x, or with b: r = b - A x (extended precision) with per-block partial sums of
// (w r)^2 (or r w r when natural) and r^2 (w = Jacobi inverse, nullptr: 1).
// Tail of the FDM refinement step fused into the residual launch (ResTail,
// count == nullptr: none).

template <int N>
__global__ void __launch_bounds__(kCgThreads) apply_kernel(const OpDev op, const double* __restrict__ x,
                                                           const double* __restrict__ b,
                                                           double* __restrict__ y,
                                                           const double* __restrict__ w,
                                                           int natural, double* __restrict__ partial,
                                                           const ResTail tail) {
  extern __shared__ double P[];
  __shared__ OpSm o;
  __shared__ double red[kCgThreads / 32][4];
  {
    const int n = N + 1;
    for (int k = threadIdx.x; k < n * n; k += kCgThreads) o.Kh[k] = op.Kh[k];
    if (op.gamma != 0.0)
      for (int k = threadIdx.x; k < n * n; k += kCgThreads) {
        o.Sv[k] = op.Sv[k];
        o.Tv[k] = op.Tv[k];
      }
    if (threadIdx.x < n) o.w[threadIdx.x] = op.w[threadIdx.x];
    if (threadIdx.x == 0) {
      o.alpha = op.alpha;
      o.beta0 = op.beta[0];
      o.beta1 = op.beta[1];
      o.gamma = op.gamma;
      o.dx = op.d[0];
      o.dy = op.d[1];
      o.G0 = op.G[0];
      o.G1 = op.G[1];
    }
    __syncthreads();
  }
  const int x0 = blockIdx.x * kCgTileX, y0 = blockIdx.y * kCgTileY;
  stage_p<N>(o, x0, y0, x, nullptr, true, 0.0, P);
  const int tx = threadIdx.x & (kCgTileX - 1), ty = threadIdx.x / kCgTileX;
  const int ux = x0 + tx, uy = y0 + ty;
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  if (ux < o.G0 && uy < o.G1) {
    const size_t k = (size_t)uy * o.G0 + ux;
    if (b) {
      const double r = residual_dd<N>(o, P, tx, ty, ux + o.dx.lo, uy + o.dy.lo, b[k]);
      y[k] = r;
      const double z = w ? r * w[k] : r;
      acc[0] = natural ? z * r : z * z;
      acc[1] = r * r;
    } else {
      y[k] = apply_n<N>(o, P, tx, ty, ux + o.dx.lo, uy + o.dy.lo);
    }
  }
  if (partial) {
    block_sum4(acc, red);
    if (threadIdx.x == 0) {
      partial[2 * (blockIdx.y * gridDim.x + blockIdx.x)] = acc[0];
      partial[2 * (blockIdx.y * gridDim.x + blockIdx.x) + 1] = acc[1];
    }
  }
  if (!tail.count) return;
  // the last block to finish sums the partials in block order and runs the
  // refinement step's convergence test (no block waits for another)
  __shared__ unsigned last;
  __threadfence();
  __syncthreads();
  const unsigned nb = gridDim.x * gridDim.y;
  if (threadIdx.x == 0) last = atomicAdd(tail.count, 1u) == nb - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  double s[4] = {0.0, 0.0, 0.0, 0.0};
  for (unsigned k = threadIdx.x; k < nb; k += kCgThreads) {
    s[0] += __ldcg(partial + 2 * k);
    s[1] += __ldcg(partial + 2 * k + 1);
  }
  block_sum4(s, red);
  if (threadIdx.x == 0) {
    tail.res[0] = s[0];
    tail.res[1] = s[1];
    *tail.count = 0u;
    fdm_check_state(tail.p, tail.st, s[0], tail.h);
  }
}

template <int N>
cudaError_t launch_apply_n(const OpDev& op, const double* x, const double* b, double* y,
                           const double* w, int natural, double* partial, const ResTail& tail,
                           cudaStream_t s) {
  dim3 grid((op.G[0] + kCgTileX - 1) / kCgTileX, (op.G[1] + kCgTileY - 1) / kCgTileY);
  const size_t smem = sizeof(double) * (size_t)Geo<N>::W * Geo<N>::H;
  apply_kernel<N><<<grid, kCgThreads, smem, s>>>(op, x, b, y, w, natural, partial, tail);
  return cudaGetLastError();
}

template <int N, int K, int LP = 0>
const void* kernel_ptr() {
  return (const void*)cg_n_kernel<N, K, LP>;
}

// lp: 0 FP64 apply (every order); 1 BF16, 2 FP16 input with FP32 arithmetic
// (orders 4 to 8).
const void* pick(int N, int K, int lp = 0) {
#define SE_CASE(n)                                         \
  case n:                                                  \
    return K > 0 ? kernel_ptr<n, kCgResidentTiles>() : kernel_ptr<n, 0>();
#define SE_LP_CASE(n, l)                                                            \
  case n:                                                                           \
    return K > 0 ? kernel_ptr<n, kCgResidentTiles, l>() : kernel_ptr<n, 0, l>();
  if (lp == 1) {
    switch (N) {
      SE_LP_CASE(4, 1) SE_LP_CASE(5, 1) SE_LP_CASE(6, 1) SE_LP_CASE(7, 1) SE_LP_CASE(8, 1)
      default:
        return nullptr;
    }
  }
  if (lp == 2) {
    switch (N) {
      SE_LP_CASE(4, 2) SE_LP_CASE(5, 2) SE_LP_CASE(6, 2) SE_LP_CASE(7, 2) SE_LP_CASE(8, 2)
      default:
        return nullptr;
    }
  }
  if (lp != 0) return nullptr;
  switch (N) {
    SE_CASE(2) SE_CASE(3) SE_CASE(4) SE_CASE(5) SE_CASE(6) SE_CASE(7) SE_CASE(8) SE_CASE(9)
    SE_CASE(10) SE_CASE(11) SE_CASE(12)
    default:
      return nullptr;
  }
#undef SE_CASE
#undef SE_LP_CASE
}

}  // namespace

#define SE_APPLY_CASE(n) \
  case n:                \
    return launch_apply_n<n>(op, x, b, y, w, natural, partial, tail, s);

namespace {
cudaError_t residual_any(const OpDev& op, const double* x, const double* b, double* y,
                         const double* w, int natural, double* partial, const ResTail& tail,
                         cudaStream_t s) {
  switch (op.d[0].N) {
    SE_APPLY_CASE(2) SE_APPLY_CASE(3) SE_APPLY_CASE(4) SE_APPLY_CASE(5) SE_APPLY_CASE(6)
    SE_APPLY_CASE(7) SE_APPLY_CASE(8) SE_APPLY_CASE(9) SE_APPLY_CASE(10) SE_APPLY_CASE(11)
    SE_APPLY_CASE(12)
    default:
      return cudaErrorInvalidValue;
  }
}
}  // namespace
#undef SE_APPLY_CASE

cudaError_t launch_residual(const OpDev& op, const double* x, const double* b, double* y,
                            const double* w, int natural, double* partial, cudaStream_t s) {
  const ResTail none{nullptr, nullptr, nullptr, nullptr, 0};
  if (b && partial && residual_ef_supported(op))
    return launch_residual_ef(op, x, b, y, w, natural, partial, none, nullptr, nullptr, 0, s);
  return residual_any(op, x, b, y, w, natural, partial, none, s);
}

cudaError_t launch_residual_check(const OpDev& op, const double* x, const double* b, double* r,
                                  const double* w, int natural, double* partial, double* res,
                                  unsigned* count, const FdmParams* p, FdmState* st,
                                  cudaGraphConditionalHandle h, cudaStream_t s, float* split_hi,
                                  float* split_lo, int split_pitch) {
  if (!partial || !count) return cudaErrorInvalidValue;
  const ResTail tail{res, count, p, st, h};
  if (residual_ef_supported(op))
    return launch_residual_ef(op, x, b, r, w, natural, partial, tail, split_hi, split_lo,
                              split_pitch, s);
  if (split_hi) {  // the general kernel, then the split
    cudaError_t e = residual_any(op, x, b, r, w, natural, partial, tail, s);
    if (e != cudaSuccess) return e;
    return launch_tc_split(r, op.G[1], op.G[0], op.G[0], split_hi, split_lo, split_pitch, s);
  }
  return residual_any(op, x, b, r, w, natural, partial, tail, s);
}


int residual_blocks(const OpDev& op) {
  return ((op.G[0] + kCgTileX - 1) / kCgTileX) * ((op.G[1] + kCgTileY - 1) / kCgTileY);
}

size_t cg_dyn_smem_bytes(int N, int nsolves) {
  return sizeof(SolveState) * nsolves + sizeof(SolveMeta) * nsolves + 16 +
         sizeof(double) * (size_t)(kCgTileX + 2 * N) * (kCgTileY + 2 * N);
}

int cg_max_grid(int device, int N, bool resident, int nsolves, int lowp) {
  const void* f = pick(N, resident ? 1 : 0, lowp);
  if (!f) return 0;
  int sms = 0, per_sm = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess)
    return 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, f, kCgThreads,
                                                    cg_dyn_smem_bytes(N, nsolves)) != cudaSuccess)
    return 0;
  return sms * per_sm;
}

cudaError_t launch_cg(const CgBatch& batch, int grid, int N, bool resident, cudaStream_t s,
                      int lowp) {
  const void* f = pick(N, resident ? 1 : 0, lowp);
  if (!f) return cudaErrorInvalidValue;
  const size_t smem = cg_dyn_smem_bytes(N, batch.nsolves);
  if (smem > 48 * 1024) {
    cudaError_t e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  void* args[] = {const_cast<CgBatch*>(&batch)};
  return cudaLaunchCooperativeKernel(f, dim3(grid), dim3(kCgThreads), args, smem, s);
}

}  // namespace seg
