// FDM products on Blackwell's fifth-generation tensor cores (tcgen05), for
// the reduced-precision fast-diagonalization inverse inside the FP64
// iterative refinement (api.cu, SE_PREC_MIXED).
//
// One product is D (M x N) = A (M x K) * B (K x N) with both operands stored
// K-contiguous ("K-major"): A as [M][K], B as [N][K], each as an FP32 pair
// hi + lo with hi exactly a TF32 number and lo the FP32 remainder. The
// product is formed as Ah Bh + Ah Bl + Al Bh (three kind::tf32 MMAs per K
// step, FP32 accumulation in tensor memory): about 21 bits of the operands'
// mantissas instead of TF32's 10, so that the refinement needs two or three
// steps instead of six to eleven.
//
// Output element (m, n) is stored at out[n * pitch + m]: the epilogue thread
// that holds accumulator row m (tensor-memory lane m) writes consecutive m
// across its warp, so every store is coalesced. The four products of one
// FDM inverse chain through this layout without any transpose
// (fdm_apply_tc in api.cu):
//   P1  T1[x'][y]  = sum_x  F[y][x]   Ex[x][x']           A = F,   B = Ex^T
//   P2  T2[y'][x'] = sum_y  T1[x'][y] Ey[y][y'] / lam     A = T1,  B = Ey^T
//   P3  T3[x][y']  = sum_x' T2[y'][x'] Ex[x][x']          A = T2,  B = Ex
//   P4  X[y][x]   += sum_y' T3[x][y'] Ey[y][y']           A = T3,  B = Ey
//
// Kernel: one CTA per 128 x BN output tile, 128 threads. Thread 0 streams the
// K blocks (32 FP32 = one 128-byte swizzle row) of A hi/lo and B hi/lo into a
// four-stage shared-memory ring by TMA (cp.async.bulk.tensor, 128-byte
// swizzle, out-of-range rows and columns zero-filled, no multicast); thread 32
// issues the MMAs (one elected thread, accumulator in tensor memory) and
// releases each stage with tcgen05.commit; then all four warps read their 32
// accumulator lanes (tcgen05.ld) and apply the epilogue. Every wait is bounded;
// a wait that gives up sets KERR_BARRIER_TIMEOUT, the CTA stores nothing,
// waits (bounded) for its MMAs in flight, frees its tensor memory and returns.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <cstring>

#include "common.cuh"

namespace seg {
namespace {

constexpr int kTcThreads = 128;
constexpr int kTcBM = 128;    // accumulator rows (tensor-memory lanes)
constexpr int kTcBK = 32;     // FP32 per K block: one 128-byte swizzle row
constexpr int kTcPolls = 1 << 22;
constexpr int kTcMaxSplit = 8;  // CTAs of one cluster sharing a tile's K range

template <int BN>
struct TcCfg {
  static constexpr int A_BYTES = kTcBM * kTcBK * 4;  // 16 KB
  static constexpr int B_BYTES = BN * kTcBK * 4;
  static constexpr int STAGE = 2 * A_BYTES + 2 * B_BYTES;
  static constexpr int STAGES = BN >= 128 ? 3 : 4;
  static constexpr int RING = STAGES * STAGE;
  static constexpr int SMEM = RING + 1024 + 256;
  static constexpr int TMEM_COLS = BN;
  // kind::tf32 instruction descriptor: D F32 (bits 4-5 = 1), A and B TF32
  // (bits 7-9 and 10-12 = 2), both K-major (bits 15, 16 = 0), N >> 3 in bits
  // 17-22, M >> 4 in bits 24-28
  static constexpr uint32_t IDESC = (1u << 4) | (2u << 7) | (2u << 10) |
                                    ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(kTcBM >> 4) << 24);
  static_assert(STAGE % 1024 == 0, "stages must keep 1024-byte alignment");
  static_assert(BN == 64 || BN == 128, "N tile");
  static_assert(SMEM <= 227 * 1024, "shared memory");
};

// The K-split exchange over the drained stage ring: this CTA's partial tile
// as CK column slices [128][W + 4] (slice p goes to cluster rank p, row 0's
// first padding float carries the sender's valid flag), then CK receive
// slots of the same shape.
template <int BN, int CK>
struct TcX {
  static constexpr int W = BN / CK;       // columns a CTA reduces and stores
  static constexpr int SP = W + 4;        // slice row pitch (floats), conflict-free float4 rows
  static constexpr int SB = kTcBM * SP * 4;  // slice bytes
  static_assert(2 * CK * SB <= TcCfg<BN>::RING, "exchange fits the ring");
};

__device__ __forceinline__ uint32_t su32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* b, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(su32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(su32(b)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t* b, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(su32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ bool mbar_wait(uint64_t* b, unsigned parity) {
  for (int i = 0; i < kTcPolls; i++)
    if (mbar_try(b, parity)) return true;
  return false;
}
__device__ __forceinline__ void tma_2d(void* dst, const CUtensorMap* map, int x, int y,
                                       uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, "
      "%3}], [%4];" ::"r"(su32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(su32(bar))
      : "memory");
}
// Shared-memory matrix descriptor of a K-major tile in the canonical 128-byte
// swizzle layout (rows of 128 bytes, 8-row groups 1024 bytes apart): start
// address >> 4 (bits 0-13), leading byte offset 16 >> 4 (bits 16-29, unused by
// this layout), stride byte offset 1024 >> 4 (bits 32-45), descriptor
// version 1 (bits 46-47), swizzle mode 2 = 128-byte (bits 61-63).
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}
__device__ __forceinline__ void mma_tf32(uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc,
                                         uint32_t accum) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(accum)
      : "memory");
}
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   su32(bar))
               : "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}

// 16 accumulator columns of this thread's lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,"
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int j = 0; j < 16; j++) v[j] = __uint_as_float(r[j]);
}

// TF32 part of x (round to nearest) and the FP32 remainder.
__device__ __forceinline__ void split_tf32(float x, float& hi, float& lo) {
  uint32_t h;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(h) : "f"(x));
  hi = __uint_as_float(h);
  lo = x - hi;
}

}  // namespace

namespace {

__device__ __forceinline__ uint32_t cluster_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
// Shared-memory address of the same location in CTA `rank` of the cluster.
__device__ __forceinline__ uint32_t cluster_addr(uint32_t saddr, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(saddr), "r"(rank));
  return r;
}
// bytes from this CTA's shared memory to another CTA's (distributed shared
// memory, the bulk-copy engine, no multicast), completing on its barrier.
__device__ __forceinline__ void bulk_to_peer(uint32_t dst, uint32_t src, uint32_t bytes,
                                             uint32_t bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.shared::cta.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          dst),
      "r"(src), "r"(bytes), "r"(bar)
      : "memory");
}

// One 128 x BN output tile per cluster of CK CTAs; CTA q of the cluster
// multiplies the q-th slice of the K blocks into its own tensor-memory
// accumulator, writes it to shared memory, and after a cluster barrier
// reduces columns [q BN / CK, (q + 1) BN / CK) of the tile over the CK
// partials (read through distributed shared memory, summed in rank order, so
// the result is deterministic) and stores them with the epilogue.
template <int BN, int CK, int EPI>
__global__ void __launch_bounds__(kTcThreads, 1)
    tc_product_kernel(const __grid_constant__ CUtensorMap mah, const __grid_constant__ CUtensorMap mal,
                      const __grid_constant__ CUtensorMap mbh, const __grid_constant__ CUtensorMap mbl,
                      const TcEpi e) {
  typedef TcCfg<BN> C;
  constexpr int S = C::STAGES;
  extern __shared__ uint8_t tc_smem_raw[];
  uint8_t* sm = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(tc_smem_raw) + 1023) &
                                           ~(uintptr_t)1023);
  uint64_t* full = reinterpret_cast<uint64_t*>(sm + C::RING);
  uint64_t* empty = full + S;
  uint64_t* done = empty + S;
  uint64_t* xbar = done + 1;  // the other ranks' slices have arrived
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(xbar + 1);
  int* abort_flag = reinterpret_cast<int*>(tmem_slot + 1);
  int* consumed_slot = abort_flag + 1;  // K blocks the MMA issuer took from the ring
  typedef TcX<BN, CK> X;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.y * kTcBM, n0 = blockIdx.x * BN;
  const int q = CK > 1 ? (int)cluster_rank() : 0;
  // this CTA's K blocks: [kb0, kb0 + nk)
  const int nkb = (e.K + kTcBK - 1) / kTcBK;
  const int per = (nkb + CK - 1) / CK;
  const int kb0 = q * per;
  const int nk = max(0, min(nkb, kb0 + per) - kb0);

  auto issue = [&](int i) {  // K block i of this CTA into stage i % S
    const int s = i % S;
    uint8_t* st = sm + s * C::STAGE;
    mbar_expect_tx(&full[s], C::STAGE);
    const int k0 = (kb0 + i) * kTcBK;
    tma_2d(st, &mah, k0, m0, &full[s]);
    tma_2d(st + C::A_BYTES, &mal, k0, m0, &full[s]);
    tma_2d(st + 2 * C::A_BYTES, &mbh, k0, n0, &full[s]);
    tma_2d(st + 2 * C::A_BYTES + C::B_BYTES, &mbl, k0, n0, &full[s]);
  };

  int issued = 0;  // producer: K blocks whose loads were issued
  if (threadIdx.x == 0) {
    for (int s = 0; s < S; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(done, 1);
    mbar_init(xbar, 1);
    *abort_flag = 0;
    *consumed_slot = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    // the first stages' loads go out before anything else
    for (; issued < nk && issued < S; issued++) issue(issued);
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     su32(tmem_slot)),
                 "r"((uint32_t)C::TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (threadIdx.x == 0) {
    // producer: the rest of this CTA's K blocks through the ring
    for (int i = issued; i < nk; i++) {
      if (!mbar_wait(&empty[i % S], ((i / S) - 1) & 1)) {
        atomicOr(e.err, (unsigned)KERR_BARRIER_TIMEOUT);
        *abort_flag = 1;
        break;
      }
      issue(i);
      issued = i + 1;
    }
  } else if (threadIdx.x == 32) {
    // MMA issuer: three TF32 products per 8-wide K step into the accumulator
    int consumed = 0;
    for (int i = 0; i < nk; i++) {
      const int s = i % S;
      if (!mbar_wait(&full[s], (i / S) & 1)) {
        atomicOr(e.err, (unsigned)KERR_BARRIER_TIMEOUT);
        *abort_flag = 1;
        break;
      }
      consumed = i + 1;
      tc_fence_after();
      const uint32_t st = su32(sm + s * C::STAGE);
      const uint64_t ah = sw128_desc(st), al = sw128_desc(st + C::A_BYTES);
      const uint64_t bh = sw128_desc(st + 2 * C::A_BYTES);
      const uint64_t bl = sw128_desc(st + 2 * C::A_BYTES + C::B_BYTES);
#pragma unroll
      for (int k = 0; k < kTcBK / 8; k++) {
        const uint64_t dk = (uint64_t)(k * 32 >> 4);  // 8 FP32 = 32 bytes along the swizzled row
        mma_tf32(tmem, ah + dk, bh + dk, C::IDESC, (i | k) != 0);
        mma_tf32(tmem, ah + dk, bl + dk, C::IDESC, 1u);
        mma_tf32(tmem, al + dk, bh + dk, C::IDESC, 1u);
      }
      mma_commit(&empty[s]);  // the stage is free once these MMAs have read it
    }
    *consumed_slot = consumed;
    mma_commit(done);  // arrives when every MMA issued so far has completed
  }
  __syncwarp();

  // the partial accumulator into shared memory (over the drained ring)
  const bool ready = mbar_wait(done, 0);
  // peers may copy into this CTA's receive slots (over its ring) once every
  // CTA of the cluster has passed this point: arrive now, wait just before
  // the copies (the arrival also publishes the barrier initialisation)
  if (CK > 1) asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");
  tc_fence_after();
  if (!ready) atomicOr(e.err, (unsigned)KERR_BARRIER_TIMEOUT);
  __syncthreads();  // the issuers' flags are visible past this barrier
  const bool mine = __syncthreads_and(ready && *abort_flag == 0);
  if (!mine && threadIdx.x == 0 && nk > 0) {
    // loads issued but never consumed may still be in flight: wait (bounded)
    // until they have landed before the ring is overwritten
    for (int i = *consumed_slot; i < issued; i++) mbar_wait(&full[i % S], (i / S) & 1);
  }
  __syncthreads();
  float* part = reinterpret_cast<float*>(sm);           // [CK][128][SP]
  float* recv = part + CK * (X::SB / 4);                // [CK][128][SP]
  {
    const int r = warp * 32 + lane;
    const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll
    for (int c = 0; c < BN; c += 16) {
      float v[16];
      if (mine && nk > 0) {
        tmem_ld16(taddr + c, v);
      } else {
#pragma unroll
        for (int j = 0; j < 16; j++) v[j] = 0.0f;
      }
#pragma unroll
      for (int j = 0; j < 16; j += 4) {
        const int col = c + j, p = col / X::W;
        *reinterpret_cast<float4*>(&part[(p * kTcBM + r) * X::SP + col - p * X::W]) =
            make_float4(v[j], v[j + 1], v[j + 2], v[j + 3]);
      }
    }
    if (r == 0)
      for (int p = 0; p < CK; p++) part[p * kTcBM * X::SP + X::W] = mine ? 1.0f : 0.0f;
  }
  bool all_ok = mine;
  if constexpr (CK > 1) {
    // slice p to rank p's receive slot q; the other ranks' slices to ours
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory");
    __syncthreads();
    if (threadIdx.x == 0) {
      mbar_expect_tx(xbar, (CK - 1) * X::SB);
      for (int p = 0; p < CK; p++) {
        if (p == q) continue;
        bulk_to_peer(cluster_addr(su32(recv + q * (X::SB / 4)), p),
                     su32(part + p * (X::SB / 4)), X::SB, cluster_addr(su32(xbar), p));
      }
    }
    const bool got = mbar_wait(xbar, 0);
    if (!got) atomicOr(e.err, (unsigned)KERR_BARRIER_TIMEOUT);
    all_ok = __syncthreads_and(got && mine);
#pragma unroll
    for (int p = 0; p < CK; p++)
      if (p != q) all_ok = all_ok && recv[p * kTcBM * X::SP + X::W] != 0.0f;
  } else {
    __syncthreads();
  }

  // this CTA's columns of the tile, summed over the cluster in rank order
  constexpr int W = X::W;
  constexpr int CH = W < 16 ? W : 16;  // columns per pass (registers)
  const int r = threadIdx.x, m = m0 + r;
  double lmv = 0.0;
  if (EPI == TC_EPI_DIVIDE && all_ok && m < e.M) lmv = e.lm[m];
  for (int c0 = q * W; all_ok && c0 < (q + 1) * W; c0 += CH) {
    // every partial's values (own slice q, the others' from the receive slots)
    float4 v[CK][CH / 4];
    const int cc = c0 - q * W;
#pragma unroll
    for (int p = 0; p < CK; p++) {
      const float* src = (p == q ? part + q * (X::SB / 4) : recv + p * (X::SB / 4)) + r * X::SP + cc;
#pragma unroll
      for (int j = 0; j < CH / 4; j++) v[p][j] = *reinterpret_cast<const float4*>(src + 4 * j);
    }
    float acc[CH];
#pragma unroll
    for (int j = 0; j < CH / 4; j++) {
      float4 t = v[0][j];
#pragma unroll
      for (int p = 1; p < CK; p++) {
        t.x += v[p][j].x;
        t.y += v[p][j].y;
        t.z += v[p][j].z;
        t.w += v[p][j].w;
      }
      acc[4 * j] = t.x;
      acc[4 * j + 1] = t.y;
      acc[4 * j + 2] = t.z;
      acc[4 * j + 3] = t.w;
    }
    if (m >= e.M) continue;
    const int nv = min(CH, e.N - (n0 + c0));  // valid columns of this pass
    if constexpr (EPI == TC_EPI_ACC64) {
      double old[CH];
#pragma unroll
      for (int j = 0; j < CH; j++)
        old[j] = j < nv ? e.out64[(size_t)(n0 + c0 + j) * e.pitch + m] : 0.0;
#pragma unroll
      for (int j = 0; j < CH; j++)
        if (j < nv) e.out64[(size_t)(n0 + c0 + j) * e.pitch + m] = old[j] + (double)acc[j];
    } else {
      double div[CH];
      if constexpr (EPI == TC_EPI_DIVIDE) {
#pragma unroll
        for (int j = 0; j < CH; j++) div[j] = j < nv ? e.ln[n0 + c0 + j] : 0.0;
      }
#pragma unroll
      for (int j = 0; j < CH; j++) {
        if (j >= nv) continue;
        float x = acc[j];
        if constexpr (EPI == TC_EPI_DIVIDE) {
          const double d = e.alpha + e.bm * lmv + e.bn * div[j];
          x = fabs(d) <= e.null_tol ? 0.0f : (float)((double)x / d);
        }
        float hi, lo;
        split_tf32(x, hi, lo);
        const size_t o = (size_t)(n0 + c0 + j) * e.pitch + m;
        e.out_hi[o] = hi;
        e.out_lo[o] = lo;
      }
    }
  }
  // no CTA leaves while a copy out of its shared memory may be in flight
  // (every rank has seen its slices arrive before it arrives here)
  if (CK > 1) {
    asm volatile("barrier.cluster.arrive.relaxed.aligned;\nbarrier.cluster.wait.aligned;" ::
                     : "memory");
  } else {
    __syncthreads();
  }
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"((uint32_t)C::TMEM_COLS)
                 : "memory");
}

// hi/lo TF32 split of an FP64 array [rows][cols] (leading dimension ld) into
// FP32 arrays with the given pitch.
__global__ void tc_split_kernel(const double* __restrict__ x, int rows, int cols, int ld,
                                float* __restrict__ hi, float* __restrict__ lo, int pitch) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int r = blockIdx.y;
  if (c >= cols) return;
  const double v = x[(size_t)r * ld + c];
  uint32_t h;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(h) : "f"((float)v));
  const float fh = __uint_as_float(h);
  hi[(size_t)r * pitch + c] = fh;
  lo[(size_t)r * pitch + c] = (float)(v - (double)fh);  // remainder of the FP64 value
}

PFN_cuTensorMapEncodeTiled_v12000 tc_encoder() {
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

// Tensor map of an FP32 [rows][pitch] operand read in boxes of 32 (K) x box_rows,
// 128-byte swizzle, zero fill outside [rows) x [cols).
bool tc_map(CUtensorMap* map, const float* p, int rows, int cols, int pitch, int box_rows) {
  PFN_cuTensorMapEncodeTiled_v12000 enc = tc_encoder();
  if (!enc || (reinterpret_cast<uintptr_t>(p) & 15) || (pitch * 4) % 16) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)pitch * 4};
  const cuuint32_t box[2] = {(cuuint32_t)kTcBK, (cuuint32_t)box_rows};
  const cuuint32_t estr[2] = {1, 1};
  std::memset(map, 0, sizeof(*map));
  return enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(p), dims, strides, box, estr,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int BN, int CK, int EPI>
cudaError_t set_smem_attr() {
  static bool attr[64] = {};
  int dev = 0;
  cudaError_t err = cudaGetDevice(&dev);
  if (err != cudaSuccess) return err;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  if (!attr[dev]) {
    err = cudaFuncSetAttribute(tc_product_kernel<BN, CK, EPI>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, TcCfg<BN>::SMEM);
    if (err != cudaSuccess) return err;
    attr[dev] = true;
  }
  return cudaSuccess;
}

cudaLaunchConfig_t tc_config(dim3 grid, int smem, int ck, cudaLaunchAttribute* at, cudaStream_t s) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = dim3(kTcThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = 1;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = ck;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cfg;
}

template <int BN, int CK, int EPI>
cudaError_t run_tc(const CUtensorMap* maps, const TcEpi& e, cudaStream_t s) {
  if (cudaError_t err = set_smem_attr<BN, CK, EPI>()) return err;
  cudaLaunchAttribute at[1];
  cudaLaunchConfig_t cfg =
      tc_config(dim3((e.N + BN - 1) / BN, (e.M + kTcBM - 1) / kTcBM, CK), TcCfg<BN>::SMEM, CK, at, s);
  return cudaLaunchKernelEx(&cfg, tc_product_kernel<BN, CK, EPI>, maps[0], maps[1], maps[2], maps[3],
                            e);
}

// Clusters of CK CTAs of the BN kernel that can be resident at once on this
// device (cached per device and shape).
template <int BN, int CK>
int max_clusters() {
  static int cache[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 1;
  if (!cache[dev]) {
    int n = 0;
    cudaLaunchAttribute at[1];
    cudaLaunchConfig_t cfg = tc_config(dim3(1, 1, CK), TcCfg<BN>::SMEM, CK, at, nullptr);
    if (set_smem_attr<BN, CK, TC_EPI_SPLIT>() != cudaSuccess ||
        cudaOccupancyMaxActiveClusters(&n, tc_product_kernel<BN, CK, TC_EPI_SPLIT>, &cfg) != cudaSuccess ||
        n < 1) {
      cudaGetLastError();
      n = 1;
    }
    cache[dev] = n;
  }
  return cache[dev];
}
int max_clusters(int bn, int ck) {
  if (bn == 64)
    return ck == 1 ? max_clusters<64, 1>() : ck == 2 ? max_clusters<64, 2>()
           : ck == 4 ? max_clusters<64, 4>() : max_clusters<64, 8>();
  return ck == 1 ? max_clusters<128, 1>() : ck == 2 ? max_clusters<128, 2>()
         : ck == 4 ? max_clusters<128, 4>() : max_clusters<128, 8>();
}

template <int BN, int EPI>
cudaError_t run_tc_ck(int ck, const CUtensorMap* maps, const TcEpi& e, cudaStream_t s) {
  if (ck == 1) return run_tc<BN, 1, EPI>(maps, e, s);
  if (ck == 2) return run_tc<BN, 2, EPI>(maps, e, s);
  if (ck == 4) return run_tc<BN, 4, EPI>(maps, e, s);
  return run_tc<BN, 8, EPI>(maps, e, s);
}

template <int EPI>
cudaError_t run_tc_shape(int bn, int ck, const CUtensorMap* maps, const TcEpi& e, cudaStream_t s) {
  if (bn == 64) return run_tc_ck<64, EPI>(ck, maps, e, s);
  return run_tc_ck<128, EPI>(ck, maps, e, s);
}

}  // namespace

// Tile shape of an M x N x K product: the N tile bn (128 or 64) and ck, the
// CTAs of one cluster that split a tile's K range (1, 2, 4 or 8), chosen for
// the most CTAs in a single wave (every cluster resident at once, at least
// one 32-wide K block per CTA); ties go to the wider tile (fewer re-reads of
// A) and then to the smaller split.
void tc_shape(int M, int N, int K, int* bn, int* ck) {
  const int mt = (M + kTcBM - 1) / kTcBM, nkb = (K + kTcBK - 1) / kTcBK;
  int best = -1;
  *bn = 128;
  *ck = 1;
  for (int b = 128; b >= 64; b /= 2) {
    const int tiles = mt * ((N + b - 1) / b);
    for (int c = 1; c <= kTcMaxSplit; c *= 2) {
      if (c > 1 && (c > nkb || tiles > max_clusters(b, c))) continue;
      const int ctas = tiles * c;
      if (ctas > best) {
        best = ctas;
        *bn = b;
        *ck = c;
      }
    }
  }
}

// Plan of D = A B with A = (a_hi + a_lo) [M][K] (pitch a_pitch) and B
// stored as (b_hi + b_lo) [N][K] (pitch b_pitch), epilogue e of kind epi:
// the tile shape and the four tensor maps, made once per buffer set.
cudaError_t tc_plan(TcPlan* p, int epi, const float* a_hi, const float* a_lo, int a_pitch,
                    const float* b_hi, const float* b_lo, int b_pitch, const TcEpi& e) {
  if (e.M <= 0 || e.N <= 0 || e.K <= 0 || !e.err) return cudaErrorInvalidValue;
  if (epi != TC_EPI_SPLIT && epi != TC_EPI_DIVIDE && epi != TC_EPI_ACC64) return cudaErrorInvalidValue;
  tc_shape(e.M, e.N, e.K, &p->bn, &p->ck);
  if (!tc_map(&p->maps[0], a_hi, e.M, e.K, a_pitch, kTcBM) ||
      !tc_map(&p->maps[1], a_lo, e.M, e.K, a_pitch, kTcBM) ||
      !tc_map(&p->maps[2], b_hi, e.N, e.K, b_pitch, p->bn) ||
      !tc_map(&p->maps[3], b_lo, e.N, e.K, b_pitch, p->bn))
    return cudaErrorInvalidValue;
  p->e = e;
  p->epi = epi;
  return cudaSuccess;
}

cudaError_t launch_tc_plan(const TcPlan& p, cudaStream_t s) {
  if (p.epi == TC_EPI_DIVIDE) return run_tc_shape<TC_EPI_DIVIDE>(p.bn, p.ck, p.maps, p.e, s);
  if (p.epi == TC_EPI_ACC64) return run_tc_shape<TC_EPI_ACC64>(p.bn, p.ck, p.maps, p.e, s);
  return run_tc_shape<TC_EPI_SPLIT>(p.bn, p.ck, p.maps, p.e, s);
}

cudaError_t launch_tc_split(const double* x, int rows, int cols, int ld, float* hi, float* lo,
                            int pitch, cudaStream_t s) {
  if (rows <= 0 || cols <= 0) return cudaErrorInvalidValue;
  const dim3 grid((cols + 255) / 256, rows);
  tc_split_kernel<<<grid, 256, 0, s>>>(x, rows, cols, ld, hi, lo, pitch);
  return cudaGetLastError();
}

}  // namespace seg
