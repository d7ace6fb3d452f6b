// Dense GEMMs of the fast-diagonalization solve (fdm.cu / api.cu), written
// for the solve's CUDA graph: one kernel launch per product, no workspace,
// no library-internal nodes, so the products can sit inside the graph's
// conditional refinement loop.
//
// C (M x N) = A (M x K) * B (K x N), all row-major with leading dimensions,
// on the tensor cores through warp-level MMA:
//   P = 0  FP64 data, m16n8k8 f64 MMA (Blackwell's FP64 tensor path; there is
//          no FP64 kind of the tcgen05 MMA), FP64 accumulation;
//   P = 1  FP32 data rounded to TF32, m16n8k8 tf32 MMA, FP32 accumulation;
//   P = 2  BF16 data, m16n8k16 bf16 MMA, FP32 accumulation.
// While a grid of 64 x 64 tiles would leave SMs idle, 32 x 32 tiles: FP64 by
// 4 warps that split each K stage and sum their partial tiles in warp order,
// low precision by 2 x 2 warps; 64 x 64 tiles (2 x 2 warps) above that. FP64
// operands stream through a multi-stage cp.async pipeline; low-precision ones pass
// through registers (converted, and the FP64 first operand scaled, on the
// way) into double-buffered shared memory. Any leading dimension (odd ones
// included) is accepted.
//
// Epilogues: store; store after the spectral divide
// C[l][k] /= alpha + bx lx[k] + by ly[l] (entries whose divisor is below
// null_tol in magnitude — the null mode — become 0); accumulate into an FP64
// C with an optional scale read from device memory. The FP64 products can
// carry the lowest k x k spectral block (k <= 8) apart from the backward
// transform: the divide moves it out of C into zlow, and the transform's
// last product adds sum_a A[r][a] U[a][c], U[a][c] = sum_b zlow[a][b]
// ex[c][b], to its outputs in double-double (the block holds the largest
// coefficients of a smooth solution, whose FP64 product rounding would
// otherwise dominate the solve's first residual).
#include <cuda_bf16.h>

#include "common.cuh"

namespace seg {
namespace {

constexpr int kThreads = 128;

template <int P>
struct Tr;
template <>
struct Tr<0> {
  typedef double S;
  typedef double Acc;
  enum { BK = 16, KS = 8, AP = 4, BP = 8 };
};
template <>
struct Tr<1> {
  typedef uint32_t S;  // TF32 bit patterns
  typedef float Acc;
  enum { BK = 32, KS = 8, AP = 4, BP = 8 };
};
template <>
struct Tr<2> {
  typedef __nv_bfloat16 S;
  typedef float Acc;
  enum { BK = 32, KS = 16, AP = 8, BP = 8 };
};

__device__ __forceinline__ double as_d(double x) { return x; }
__device__ __forceinline__ float as_f(float x) { return x; }
__device__ __forceinline__ float as_f(__nv_bfloat16 x) { return __bfloat162float(x); }

__device__ __forceinline__ uint32_t to_tf32(float f) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(f));
  return r;
}

// Element of an operand in the shared-memory type of precision P; `scale`
// multiplies FP64 inputs (the FDM's 1/max|r| normalisation).
template <int P, class T>
__device__ __forceinline__ typename Tr<P>::S to_s(T x, double scale) {
  if constexpr (P == 0) {
    return as_d(x) * scale;
  } else {
    float f;
    if constexpr (sizeof(T) == 8)
      f = (float)(as_d(x) * scale);
    else
      f = as_f(x);
    if constexpr (P == 1)
      return to_tf32(f);
    else
      return __float2bfloat16_rn(f);
  }
}

__device__ __forceinline__ void mma_f64(double (&c)[4], const double (&a)[4], const double (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}
__device__ __forceinline__ void mma_tf32(float (&c)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}
__device__ __forceinline__ void mma_bf16(float (&c)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__device__ __forceinline__ uint32_t pack_bf16(__nv_bfloat16 lo, __nv_bfloat16 hi) {
  return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

template <class TA, class TB, class TC>
struct GemmArgs {
  const TA* A;
  const TB* B;
  TC* C;
  int M, N, K, lda, ldb, ldc;
  const double* amax;  // A scale 1/max (FP64 A only), nullptr: 1
  const double* cmax;  // accumulate scale, nullptr: 1
  const double *lx, *ly;
  double alpha, bx, by, null_tol;
  // FP64 only: the low spectral block carried apart (FdmLow, common.cuh);
  // lowk = 0: none
  double* zlow;
  const double* ex;
  int ldex, lowk;
  // FP64 plain stores: when *gate != 0 (a refinement loop that has already
  // decided) the product is stored as zero; nullptr: no gate
  const int* gate;
};

enum { EPI_STORE = 0, EPI_DIVIDE = 1, EPI_ACCUM = 2 };

// Low-precision products (P = 1, 2): BM x BN block tile of 2 x 2 warps,
// operands converted (and the FP64 first operand scaled) on the way from
// global memory through registers into double-buffered shared memory.
template <int P, int kBM, int kBN, class TA, class TB, class TC, int EPI>
__global__ void __launch_bounds__(kThreads) fdm_gemm_kernel(const GemmArgs<TA, TB, TC> g) {
  typedef typename Tr<P>::S S;
  typedef typename Tr<P>::Acc Acc;
  constexpr int BK = Tr<P>::BK, KS = Tr<P>::KS;
  constexpr int AS = BK + Tr<P>::AP, BS = kBN + Tr<P>::BP;
  constexpr int AE = kBM * BK / kThreads, BE = BK * kBN / kThreads;
  constexpr int MT = kBM / 32, NT = kBN / 16;  // m16n8 tiles per warp
  __shared__ __align__(16) S As[2][kBM * AS];
  __shared__ __align__(16) S Bs[2][BK * BS];

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int gq = lane >> 2, tq = lane & 3;
  const int wm = (warp >> 1) * (kBM / 2), wn = (warp & 1) * (kBN / 2);
  const int m0 = blockIdx.y * kBM, n0 = blockIdx.x * kBN;
  double ascale = 1.0;
  if (g.amax) {
    const double m = *g.amax;
    ascale = m > 0.0 ? 1.0 / m : 0.0;
  }

  S ra[AE], rb[BE];
  auto load = [&](int k0) {
#pragma unroll
    for (int r = 0; r < AE; r++) {
      const int e = tid + r * kThreads;
      const int row = e / BK, col = e % BK;
      const int gr = m0 + row, gc = k0 + col;
      ra[r] = (gr < g.M && gc < g.K) ? to_s<P>(g.A[(size_t)gr * g.lda + gc], ascale)
                                     : to_s<P>(0.0, 1.0);
    }
#pragma unroll
    for (int r = 0; r < BE; r++) {
      const int e = tid + r * kThreads;
      const int row = e / kBN, col = e % kBN;
      const int gr = k0 + row, gc = n0 + col;
      rb[r] = (gr < g.K && gc < g.N) ? to_s<P>(g.B[(size_t)gr * g.ldb + gc], 1.0) : to_s<P>(0.0, 1.0);
    }
  };
  auto store = [&](int buf) {
#pragma unroll
    for (int r = 0; r < AE; r++) {
      const int e = tid + r * kThreads;
      As[buf][(e / BK) * AS + e % BK] = ra[r];
    }
#pragma unroll
    for (int r = 0; r < BE; r++) {
      const int e = tid + r * kThreads;
      Bs[buf][(e / kBN) * BS + e % kBN] = rb[r];
    }
  };

  Acc acc[MT][NT][4];
#pragma unroll
  for (int i = 0; i < MT; i++)
#pragma unroll
    for (int j = 0; j < NT; j++)
#pragma unroll
      for (int q = 0; q < 4; q++) acc[i][j][q] = Acc(0);

  const int KT = (g.K + BK - 1) / BK;
  load(0);
  store(0);
  __syncthreads();
  for (int kt = 0; kt < KT; kt++) {
    const int buf = kt & 1;
    if (kt + 1 < KT) load((kt + 1) * BK);
    const S* as = As[buf];
    const S* bs = Bs[buf];
#pragma unroll
    for (int kk = 0; kk < BK; kk += KS) {
      if constexpr (P == 0 || P == 1) {
        S a[MT][4], b[NT][2];
#pragma unroll
        for (int mt = 0; mt < MT; mt++) {
          const int r0 = wm + mt * 16 + gq;
          a[mt][0] = as[r0 * AS + kk + tq];
          a[mt][1] = as[(r0 + 8) * AS + kk + tq];
          a[mt][2] = as[r0 * AS + kk + tq + 4];
          a[mt][3] = as[(r0 + 8) * AS + kk + tq + 4];
        }
#pragma unroll
        for (int nt = 0; nt < NT; nt++) {
          const int c0 = wn + nt * 8 + gq;
          b[nt][0] = bs[(kk + tq) * BS + c0];
          b[nt][1] = bs[(kk + tq + 4) * BS + c0];
        }
#pragma unroll
        for (int mt = 0; mt < MT; mt++)
#pragma unroll
          for (int nt = 0; nt < NT; nt++) {
            if constexpr (P == 0)
              mma_f64(acc[mt][nt], a[mt], b[nt]);
            else
              mma_tf32(acc[mt][nt], a[mt], b[nt]);
          }
      } else {
        uint32_t a[MT][4], b[NT][2];
#pragma unroll
        for (int mt = 0; mt < MT; mt++) {
          const int r0 = wm + mt * 16 + gq;
          a[mt][0] = *reinterpret_cast<const uint32_t*>(&as[r0 * AS + kk + 2 * tq]);
          a[mt][1] = *reinterpret_cast<const uint32_t*>(&as[(r0 + 8) * AS + kk + 2 * tq]);
          a[mt][2] = *reinterpret_cast<const uint32_t*>(&as[r0 * AS + kk + 2 * tq + 8]);
          a[mt][3] = *reinterpret_cast<const uint32_t*>(&as[(r0 + 8) * AS + kk + 2 * tq + 8]);
        }
#pragma unroll
        for (int nt = 0; nt < NT; nt++) {
          const int c0 = wn + nt * 8 + gq;
          b[nt][0] = pack_bf16(bs[(kk + 2 * tq) * BS + c0], bs[(kk + 2 * tq + 1) * BS + c0]);
          b[nt][1] = pack_bf16(bs[(kk + 2 * tq + 8) * BS + c0], bs[(kk + 2 * tq + 9) * BS + c0]);
        }
#pragma unroll
        for (int mt = 0; mt < MT; mt++)
#pragma unroll
          for (int nt = 0; nt < NT; nt++) mma_bf16(acc[mt][nt], a[mt], b[nt]);
      }
    }
    if (kt + 1 < KT) store(buf ^ 1);
    __syncthreads();
  }

  double cscale = 1.0;
  if (EPI == EPI_ACCUM && g.cmax) cscale = *g.cmax;
#pragma unroll
  for (int mt = 0; mt < MT; mt++)
#pragma unroll
    for (int nt = 0; nt < NT; nt++)
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int r = m0 + wm + mt * 16 + gq + 8 * h;
        if (r >= g.M) continue;
#pragma unroll
        for (int q = 0; q < 2; q++) {
          const int c = n0 + wn + nt * 8 + 2 * tq + q;
          if (c >= g.N) continue;
          double v = (double)acc[mt][nt][2 * h + q];
          TC* dst = g.C + (size_t)r * g.ldc + c;
          if constexpr (EPI == EPI_DIVIDE) {
            const double d = g.alpha + g.bx * g.lx[c] + g.by * g.ly[r];
            v = fabs(d) <= g.null_tol ? 0.0 : v / d;
          }
          if constexpr (EPI == EPI_ACCUM) {
            *dst += v * cscale;
          } else {
            if constexpr (sizeof(TC) == 8)
              *dst = v;
            else if constexpr (sizeof(TC) == 4)
              *dst = (float)v;
            else
              *dst = __float2bfloat16_rn((float)v);
          }
        }
      }
}

// ---------------------------------------------------------------------------
// FP64 products: multi-stage cp.async pipeline (8-byte copies with zero fill,
// so any leading dimension and any edge), BM x BN block tile of WM x WN
// warps, each warp (BM/WM) x (BN/WN) in m16n8 MMA tiles.
//
constexpr int kLowMax = 8;
// Shared-memory doubles of the low block of a BM x BN output tile: zlow
// (8 x 8), the tile's rows of A's first 8 columns, U (8 x BN) as hi and lo.
template <int BM, int BN>
struct LowSm {
  static constexpr int SIZE = kLowMax * kLowMax + BM * kLowMax + 2 * kLowMax * BN;
};

template <int BM_, int BN_, int WM_, int WN_, int ST_, int BK_ = 16>
struct DCfg {
  static constexpr int BM = BM_, BN = BN_, WM = WM_, WN = WN_, ST = ST_;
  static constexpr int BK = BK_, AS = BK + 4, BS = BN + 8;
  static constexpr int THREADS = WM * WN * 32;
  static constexpr int MT = BM / WM / 16, NT = BN / WN / 8;
  static constexpr int A_ELEMS = BM * AS, B_ELEMS = BK * BS;
  static constexpr size_t SMEM = (size_t)ST * (A_ELEMS + B_ELEMS) * sizeof(double);
  static_assert(ST * (A_ELEMS + B_ELEMS) >= LowSm<BM, BN>::SIZE, "low block exceeds the pipeline");
};

__device__ __forceinline__ void cp_async8(void* smem, const void* gmem, bool valid) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(gmem),
               "r"(valid ? 8 : 0));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// The low block's global operands of one thread, loaded into registers when
// the kernel starts (they do not depend on the product), so their latency
// hides behind the main loop: one zlow entry, this thread's share of A's
// first 8 columns over the tile's rows, and the 8 leading entries of the
// ex row of the output column whose U entries this thread forms (entries
// tid, tid + THREADS, ... of the 8 x BN block, all in column tid % BN).
template <int BM, int BN, int THREADS>
struct LowRegs {
  static_assert(THREADS % BN == 0 && THREADS >= kLowMax * kLowMax, "low block thread map");
  static constexpr int AL = (BM * kLowMax + THREADS - 1) / THREADS;
  static constexpr int UE = kLowMax * BN / THREADS;
  double z, al[AL], ex[kLowMax];
};

template <int BM, int BN, int THREADS>
__device__ __forceinline__ void low_prefetch(const GemmArgs<double, double, double>& g, int m0,
                                             int n0, int tid, LowRegs<BM, BN, THREADS>& L) {
  const int lk = g.lowk;
  {
    const int a = tid / kLowMax, b = tid % kLowMax;  // zlow entry (a, b) as an 8 x 8 block
    L.z = (tid < kLowMax * kLowMax && a < lk && b < lk) ? g.zlow[a * lk + b] : 0.0;
  }
#pragma unroll
  for (int q = 0; q < LowRegs<BM, BN, THREADS>::AL; q++) {
    const int e = tid + q * THREADS, r = e / kLowMax, a = e % kLowMax, gr = m0 + r;
    L.al[q] = (e < BM * kLowMax && a < lk && gr < g.M) ? g.A[(size_t)gr * g.lda + a] : 0.0;
  }
  const int gc = n0 + tid % BN;
#pragma unroll
  for (int b = 0; b < kLowMax; b++)
    L.ex[b] = (b < lk && gc < g.N) ? g.ex[(size_t)gc * g.ldex + b] : 0.0;
}

// Writes the prefetched operands to sm (LowSm layout: zlow as 8 x 8 padded
// with zeros, A's rows, U hi and lo) and forms U there; ends with the block
// synchronised.
template <int BM, int BN, int THREADS>
__device__ __forceinline__ void low_stage(double* sm, int tid, const LowRegs<BM, BN, THREADS>& L) {
  double* zl = sm;
  double* al = zl + kLowMax * kLowMax;
  double* uh = al + BM * kLowMax;
  double* ul = uh + kLowMax * BN;
  if (tid < kLowMax * kLowMax) zl[tid] = L.z;
#pragma unroll
  for (int q = 0; q < LowRegs<BM, BN, THREADS>::AL; q++) {
    const int e = tid + q * THREADS;
    if (e < BM * kLowMax) al[e] = L.al[q];
  }
  __syncthreads();
  const int c = tid % BN;
#pragma unroll
  for (int q = 0; q < LowRegs<BM, BN, THREADS>::UE; q++) {
    const int a = (tid + q * THREADS) / BN;
    double h = 0.0, l = 0.0;
#pragma unroll
    for (int b = 0; b < kLowMax; b++) dd_fma(h, l, zl[a * kLowMax + b], L.ex[b]);
    uh[a * BN + c] = h;
    ul[a * BN + c] = l;
  }
  __syncthreads();
}

// v (the product's FP64 output at tile row r, column c) plus the low block,
// plus the old value when accumulating, rounded once. Entries beyond lowk
// are zero in sm, so the sums run over all 8.
template <int BM, int BN, int EPI>
__device__ __forceinline__ double low_add(const double* sm, int r, int c, double v,
                                          const double* dst) {
  const double* al = sm + kLowMax * kLowMax + r * kLowMax;
  const double* uh = sm + kLowMax * kLowMax + BM * kLowMax;
  const double* ul = uh + kLowMax * BN;
  double h = 0.0, l = 0.0;
#pragma unroll
  for (int a = 0; a < kLowMax; a++) {
    dd_fma(h, l, al[a], uh[a * BN + c]);
    l = fma(al[a], ul[a * BN + c], l);
  }
  dd_add(h, l, v);
  if constexpr (EPI == EPI_ACCUM) dd_add(h, l, *dst);
  return h + l;
}

template <class C, int EPI>
__global__ void __launch_bounds__(C::THREADS) fdm_dgemm_kernel(const GemmArgs<double, double, double> g) {
  extern __shared__ __align__(16) double dsm[];
  double* As = dsm;
  double* Bs = dsm + C::ST * C::A_ELEMS;
  const bool closed = EPI == EPI_STORE && g.gate && *g.gate != 0;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int gq = lane >> 2, tq = lane & 3;
  const int wm = (warp / C::WN) * (C::BM / C::WM), wn = (warp % C::WN) * (C::BN / C::WN);
  const int m0 = blockIdx.y * C::BM, n0 = blockIdx.x * C::BN;
  const int nkt = (g.K + C::BK - 1) / C::BK;
  LowRegs<C::BM, C::BN, C::THREADS> LR;
  if constexpr (EPI != EPI_DIVIDE) {
    if (g.lowk) low_prefetch<C::BM, C::BN, C::THREADS>(g, m0, n0, tid, LR);
  }

  auto issue = [&](int i) {
    const int k0 = i * C::BK;
    double* as = As + (i % C::ST) * C::A_ELEMS;
    double* bs = Bs + (i % C::ST) * C::B_ELEMS;
#pragma unroll
    for (int e = tid; e < C::BM * C::BK; e += C::THREADS) {
      const int row = e / C::BK, col = e % C::BK;
      const int gr = m0 + row, gc = k0 + col;
      const bool ok = gr < g.M && gc < g.K;
      cp_async8(as + row * C::AS + col, ok ? g.A + (size_t)gr * g.lda + gc : g.A, ok);
    }
#pragma unroll
    for (int e = tid; e < C::BK * C::BN; e += C::THREADS) {
      const int row = e / C::BN, col = e % C::BN;
      const int gr = k0 + row, gc = n0 + col;
      const bool ok = gr < g.K && gc < g.N;
      cp_async8(bs + row * C::BS + col, ok ? g.B + (size_t)gr * g.ldb + gc : g.B, ok);
    }
  };

  double acc[C::MT][C::NT][4];
#pragma unroll
  for (int i = 0; i < C::MT; i++)
#pragma unroll
    for (int j = 0; j < C::NT; j++)
#pragma unroll
      for (int q = 0; q < 4; q++) acc[i][j][q] = 0.0;

#pragma unroll
  for (int s = 0; s < C::ST - 1; s++) {
    if (s < nkt) issue(s);
    cp_async_commit();
  }
  for (int i = 0; i < nkt; i++) {
    cp_async_wait<C::ST - 2>();
    __syncthreads();
    if (i + C::ST - 1 < nkt) issue(i + C::ST - 1);
    cp_async_commit();
    const double* as = As + (i % C::ST) * C::A_ELEMS;
    const double* bs = Bs + (i % C::ST) * C::B_ELEMS;
#pragma unroll
    for (int kk = 0; kk < C::BK; kk += 8) {
      double a[C::MT][4], b[C::NT][2];
#pragma unroll
      for (int mt = 0; mt < C::MT; mt++) {
        const int r0 = wm + mt * 16 + gq;
        a[mt][0] = as[r0 * C::AS + kk + tq];
        a[mt][1] = as[(r0 + 8) * C::AS + kk + tq];
        a[mt][2] = as[r0 * C::AS + kk + tq + 4];
        a[mt][3] = as[(r0 + 8) * C::AS + kk + tq + 4];
      }
#pragma unroll
      for (int nt = 0; nt < C::NT; nt++) {
        const int c0 = wn + nt * 8 + gq;
        b[nt][0] = bs[(kk + tq) * C::BS + c0];
        b[nt][1] = bs[(kk + tq + 4) * C::BS + c0];
      }
#pragma unroll
      for (int mt = 0; mt < C::MT; mt++)
#pragma unroll
        for (int nt = 0; nt < C::NT; nt++) mma_f64(acc[mt][nt], a[mt], b[nt]);
    }
  }
  cp_async_wait<0>();
  const int lk = g.lowk;
  if constexpr (EPI != EPI_DIVIDE) {
    if (lk) {
      __syncthreads();  // the pipeline's shared memory is free from here
      low_stage<C::BM, C::BN, C::THREADS>(dsm, tid, LR);
    }
  }

#pragma unroll
  for (int mt = 0; mt < C::MT; mt++)
#pragma unroll
    for (int nt = 0; nt < C::NT; nt++)
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int r = m0 + wm + mt * 16 + gq + 8 * h;
        if (r >= g.M) continue;
#pragma unroll
        for (int q = 0; q < 2; q++) {
          const int c = n0 + wn + nt * 8 + 2 * tq + q;
          if (c >= g.N) continue;
          double v = acc[mt][nt][2 * h + q];
          double* dst = g.C + (size_t)r * g.ldc + c;
          if constexpr (EPI == EPI_DIVIDE) {
            const double d = g.alpha + g.bx * g.lx[c] + g.by * g.ly[r];
            v = fabs(d) <= g.null_tol ? 0.0 : v / d;
            if (r < lk && c < lk) {
              g.zlow[r * lk + c] = v;
              v = 0.0;
            }
          } else {
            if (lk) {
              *dst = low_add<C::BM, C::BN, EPI>(dsm, r - m0, c - n0, v, dst);
              continue;
            }
          }
          if constexpr (EPI == EPI_ACCUM)
            *dst += v;
          else
            *dst = closed ? 0.0 : v;
        }
      }
}

template <class C, int EPI>
cudaError_t run_d(const GemmArgs<double, double, double>& g, cudaStream_t s) {
  if (g.M <= 0 || g.N <= 0 || g.K <= 0) return cudaErrorInvalidValue;
  if (C::SMEM > 48 * 1024) {
    static bool attr[64] = {};  // per kernel instantiation and device
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (!attr[dev]) {
      e = cudaFuncSetAttribute(fdm_dgemm_kernel<C, EPI>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)C::SMEM);
      if (e != cudaSuccess) return e;
      attr[dev] = true;
    }
  }
  const dim3 grid((g.N + C::BN - 1) / C::BN, (g.M + C::BM - 1) / C::BM);
  fdm_dgemm_kernel<C, EPI><<<grid, C::THREADS, C::SMEM, s>>>(g);
  return cudaGetLastError();
}

// FP64 products split over K inside the block: a 32 x 32 output tile per
// block of W warps; stage i holds a (8 W KW)-wide slice of K and warp w
// multiplies its w-th (8 KW)-wide part, so every warp keeps the whole tile's
// 8 accumulator fragments (8 independent MMA chains) and runs 8 KW MMAs
// between barriers. At the end the W partial tiles are summed through shared
// memory in warp order (deterministic) and the epilogue is applied.
template <int W_, int ST_, int KW_ = 1>
struct KCfg {
  static constexpr int W = W_, ST = ST_, KW = KW_;
  static constexpr int BM = 32, BN = 32, BK = 8 * W * KW;
  static constexpr int AS = BK + 4, BS = BN + 4, RS = BN + 1;
  static constexpr int THREADS = 32 * W;
  static constexpr int A_ELEMS = BM * AS, B_ELEMS = BK * BS;
  static constexpr int PIPE = ST * (A_ELEMS + B_ELEMS), RED = W * BM * RS;
  static constexpr int LOW = RED + LowSm<BM, BN>::SIZE;  // partial tiles, then the low block
  static constexpr size_t SMEM = sizeof(double) * (size_t)(PIPE > LOW ? PIPE : LOW);
};

template <class C, int EPI>
__global__ void __launch_bounds__(C::THREADS) fdm_dgemm_ksplit_kernel(
    const GemmArgs<double, double, double> g) {
  extern __shared__ __align__(16) double dsm[];
  double* As = dsm;
  double* Bs = dsm + C::ST * C::A_ELEMS;
  const bool closed = EPI == EPI_STORE && g.gate && *g.gate != 0;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int gq = lane >> 2, tq = lane & 3;
  const int m0 = blockIdx.y * C::BM, n0 = blockIdx.x * C::BN;
  const int nkt = (g.K + C::BK - 1) / C::BK;
  LowRegs<C::BM, C::BN, C::THREADS> LR;
  if constexpr (EPI != EPI_DIVIDE) {
    if (g.lowk) low_prefetch<C::BM, C::BN, C::THREADS>(g, m0, n0, tid, LR);
  }

  auto issue = [&](int i) {
    const int k0 = i * C::BK;
    double* as = As + (i % C::ST) * C::A_ELEMS;
    double* bs = Bs + (i % C::ST) * C::B_ELEMS;
#pragma unroll
    for (int e = tid; e < C::BM * C::BK; e += C::THREADS) {
      const int row = e / C::BK, col = e % C::BK;
      const int gr = m0 + row, gc = k0 + col;
      const bool ok = gr < g.M && gc < g.K;
      cp_async8(as + row * C::AS + col, ok ? g.A + (size_t)gr * g.lda + gc : g.A, ok);
    }
#pragma unroll
    for (int e = tid; e < C::BK * C::BN; e += C::THREADS) {
      const int row = e / C::BN, col = e % C::BN;
      const int gr = k0 + row, gc = n0 + col;
      const bool ok = gr < g.K && gc < g.N;
      cp_async8(bs + row * C::BS + col, ok ? g.B + (size_t)gr * g.ldb + gc : g.B, ok);
    }
  };

  double acc[2][4][4];
#pragma unroll
  for (int i = 0; i < 2; i++)
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
      for (int q = 0; q < 4; q++) acc[i][j][q] = 0.0;

#pragma unroll
  for (int s = 0; s < C::ST - 1; s++) {
    if (s < nkt) issue(s);
    cp_async_commit();
  }
  for (int i = 0; i < nkt; i++) {
    cp_async_wait<C::ST - 2>();
    __syncthreads();
    if (i + C::ST - 1 < nkt) issue(i + C::ST - 1);
    cp_async_commit();
    const double* as = As + (i % C::ST) * C::A_ELEMS;
    const double* bs = Bs + (i % C::ST) * C::B_ELEMS;
#pragma unroll
    for (int ks = 0; ks < C::KW; ks++) {
      const int kk = (warp * C::KW + ks) * 8;
      double a[2][4], b[4][2];
#pragma unroll
      for (int mt = 0; mt < 2; mt++) {
        const int r0 = mt * 16 + gq;
        a[mt][0] = as[r0 * C::AS + kk + tq];
        a[mt][1] = as[(r0 + 8) * C::AS + kk + tq];
        a[mt][2] = as[r0 * C::AS + kk + tq + 4];
        a[mt][3] = as[(r0 + 8) * C::AS + kk + tq + 4];
      }
#pragma unroll
      for (int nt = 0; nt < 4; nt++) {
        const int c0 = nt * 8 + gq;
        b[nt][0] = bs[(kk + tq) * C::BS + c0];
        b[nt][1] = bs[(kk + tq + 4) * C::BS + c0];
      }
#pragma unroll
      for (int mt = 0; mt < 2; mt++)
#pragma unroll
        for (int nt = 0; nt < 4; nt++) mma_f64(acc[mt][nt], a[mt], b[nt]);
    }
  }
  cp_async_wait<0>();
  __syncthreads();

  // partial tiles of the W warps, summed in warp order
  double* red = dsm;
#pragma unroll
  for (int mt = 0; mt < 2; mt++)
#pragma unroll
    for (int nt = 0; nt < 4; nt++)
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const int r = mt * 16 + gq + (q >> 1) * 8, c = nt * 8 + 2 * tq + (q & 1);
        red[(warp * C::BM + r) * C::RS + c] = acc[mt][nt][q];
      }
  const int lk = g.lowk;
  if constexpr (EPI != EPI_DIVIDE) {
    if (lk) low_stage<C::BM, C::BN, C::THREADS>(dsm + C::RED, tid, LR);
  }
  __syncthreads();
  for (int e = tid; e < C::BM * C::BN; e += C::THREADS) {
    const int r = e / C::BN, c = e % C::BN;
    const int gr = m0 + r, gc = n0 + c;
    if (gr >= g.M || gc >= g.N) continue;
    double v = red[r * C::RS + c];
#pragma unroll
    for (int w = 1; w < C::W; w++) v += red[(w * C::BM + r) * C::RS + c];
    double* dst = g.C + (size_t)gr * g.ldc + gc;
    if constexpr (EPI == EPI_DIVIDE) {
      const double d = g.alpha + g.bx * g.lx[gc] + g.by * g.ly[gr];
      v = fabs(d) <= g.null_tol ? 0.0 : v / d;
      if (gr < lk && gc < lk) {
        g.zlow[gr * lk + gc] = v;
        v = 0.0;
      }
    } else {
      if (lk) {
        *dst = low_add<C::BM, C::BN, EPI>(dsm + C::RED, r, c, v, dst);
        continue;
      }
    }
    if constexpr (EPI == EPI_ACCUM)
      *dst += v;
    else
      *dst = closed ? 0.0 : v;
  }
}

template <class C, int EPI>
cudaError_t run_k(const GemmArgs<double, double, double>& g, cudaStream_t s) {
  if (g.M <= 0 || g.N <= 0 || g.K <= 0) return cudaErrorInvalidValue;
  if (C::SMEM > 48 * 1024) {
    static bool attr[64] = {};  // per kernel instantiation and device
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (!attr[dev]) {
      e = cudaFuncSetAttribute(fdm_dgemm_ksplit_kernel<C, EPI>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM);
      if (e != cudaSuccess) return e;
      attr[dev] = true;
    }
  }
  const dim3 grid((g.N + C::BN - 1) / C::BN, (g.M + C::BM - 1) / C::BM);
  fdm_dgemm_ksplit_kernel<C, EPI><<<grid, C::THREADS, C::SMEM, s>>>(g);
  return cudaGetLastError();
}

// Tile shape by problem size: 32 x 32 tiles (four times the blocks) until
// the 64 x 64 grid alone covers the GPU's 148 SMs.
inline bool small_tiles(int M, int N) { return ((M + 63) / 64) * ((N + 63) / 64) < 148; }

template <int P, class TA, class TB, class TC, int EPI>
cudaError_t run(const GemmArgs<TA, TB, TC>& g, cudaStream_t s) {
  if (g.M <= 0 || g.N <= 0 || g.K <= 0) return cudaErrorInvalidValue;
  if constexpr (P == 0) {
    if (small_tiles(g.M, g.N)) return run_k<KCfg<4, 3>, EPI>(g, s);
    return run_d<DCfg<64, 64, 2, 2, 3>, EPI>(g, s);
  } else {
    if (small_tiles(g.M, g.N)) {
      const dim3 grid((g.N + 31) / 32, (g.M + 31) / 32);
      fdm_gemm_kernel<P, 32, 32, TA, TB, TC, EPI><<<grid, kThreads, 0, s>>>(g);
    } else {
      const dim3 grid((g.N + 63) / 64, (g.M + 63) / 64);
      fdm_gemm_kernel<P, 64, 64, TA, TB, TC, EPI><<<grid, kThreads, 0, s>>>(g);
    }
    return cudaGetLastError();
  }
}

}  // namespace

// prec: 0 FP64, 1 TF32 on FP32 data, 2 BF16. Types by role:
//  in:  FP64 (prec 0, or the normalised first product of prec 1/2 when amax
//       is given), else the low type;
//  out: FP64 for accumulate, else the precision's type.
cudaError_t launch_fdm_gemm(int prec, int epi, const void* A, int a_fp64, const void* B, void* C,
                            int c_fp64, int M, int N, int K, int lda, int ldb, int ldc,
                            const double* amax, const double* cmax, const double* lx,
                            const double* ly, double alpha, double bx, double by, double null_tol,
                            cudaStream_t s, const FdmLow* low, const int* gate) {
#define SE_GEMM_ARGS(TA, TB, TC)                                                              \
  GemmArgs<TA, TB, TC> g{(const TA*)A, (const TB*)B, (TC*)C, M, N, K, lda, ldb, ldc, amax, cmax, \
                         lx, ly, alpha, bx, by, null_tol, nullptr, nullptr, 0, 0, nullptr}
  if (prec == 0) {
    SE_GEMM_ARGS(double, double, double);
    g.gate = gate;
    if (low && low->k > 0) {
      if (low->k > kLowMax || !low->zlow || (epi != EPI_DIVIDE && !low->ex))
        return cudaErrorInvalidValue;
      g.zlow = low->zlow;
      g.ex = low->ex;
      g.ldex = low->ldex;
      g.lowk = low->k;
    }
    if (epi == EPI_DIVIDE) return run<0, double, double, double, EPI_DIVIDE>(g, s);
    if (epi == EPI_ACCUM) return run<0, double, double, double, EPI_ACCUM>(g, s);
    return run<0, double, double, double, EPI_STORE>(g, s);
  }
  if (prec == 1) {
    if (a_fp64) {
      SE_GEMM_ARGS(double, float, float);
      return run<1, double, float, float, EPI_STORE>(g, s);
    }
    if (c_fp64) {
      SE_GEMM_ARGS(float, float, double);
      return run<1, float, float, double, EPI_ACCUM>(g, s);
    }
    SE_GEMM_ARGS(float, float, float);
    if (epi == EPI_DIVIDE) return run<1, float, float, float, EPI_DIVIDE>(g, s);
    return run<1, float, float, float, EPI_STORE>(g, s);
  }
  typedef __nv_bfloat16 bf;
  if (a_fp64) {
    SE_GEMM_ARGS(double, bf, bf);
    return run<2, double, bf, bf, EPI_STORE>(g, s);
  }
  if (c_fp64) {
    SE_GEMM_ARGS(bf, bf, double);
    return run<2, bf, bf, double, EPI_ACCUM>(g, s);
  }
  SE_GEMM_ARGS(bf, bf, bf);
  if (epi == EPI_DIVIDE) return run<2, bf, bf, bf, EPI_DIVIDE>(g, s);
  return run<2, bf, bf, bf, EPI_STORE>(g, s);
#undef SE_GEMM_ARGS
}

}  // namespace seg
