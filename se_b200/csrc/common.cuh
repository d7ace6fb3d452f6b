// Internal declarations shared by the segpu CUDA sources (not installed).
//
// Device data layout
//  - Field values: double[nVertsTotal][ndofs] in the reference's vertex
//    order (x fastest, periodic duplicates stored), so that host uploads and
//    downloads are single copies and the SL gathers read an element's
//    (N+1)^2 block as N+1 contiguous rows of N+1 values.
//  - Solver vectors ("unknowns"): the reference's vector ordering, which on
//    SE's regular Cartesian meshes is always a row-major rectangle of the
//    vertex grid: rows [lo_y, hi_y), columns [lo_x, hi_x). Dirichlet and
//    periodic-duplicate vertices are not unknowns.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

#define SE_MAXN 12
#define SE_MAXN1 (SE_MAXN + 1)

namespace seg {

// Everything a kernel needs to know about one mesh (passed by value; lives
// in the kernel parameter bank).
struct MeshDev {
  int N;
  int nEls[2];
  int nVerts[2];
  int periodic[2];
  double min[2], max[2], dx[2];
  double two_over_dx[2];  // 2.0/dx, rounded as the reference rounds it
  double span[2];         // max - min
  double nspan[2];        // min - max
  double abcissa[SE_MAXN1];
  double lambda[SE_MAXN1];  // 1 / prod_{k != j} (x_j - x_k): Lagrange product weights
  double w[SE_MAXN1];       // GLL weights
  double dC[SE_MAXN1 * SE_MAXN1];  // cardinal derivative matrix, row = point
};

// One direction of the tensor-product operator on the unknown grid.
struct Dir {
  int nE, N, nV;
  int periodic;
  int lo, hi;  // unknown vertex range [lo, hi)
};

// A = alpha (W x W) + beta[0] (Kx x W) + beta[1] (W x Ky): the assembled
// c*Mass + s*Laplacian of SE on a uniform Cartesian GLL mesh, with Kh the
// 1-D reference-element stiffness and W the assembled 1-D GLL weights.
struct OpDev {
  Dir d[2];
  int G[2];  // unknowns per direction
  double alpha;
  double beta[2];
  double Kh[SE_MAXN1 * SE_MAXN1];
  double w[SE_MAXN1];
  // Spectral vanishing viscosity (HelmholtzEqn with svvCutoff != 0):
  // + gamma (Sv along x (x) Tv along y), the assembled 1-D element matrices
  // S = (F D)^T diag(w) (F D) and T = F^T diag(w) F of the modal filter F;
  // gamma == 0: no such term (and Sv, Tv unused).
  double gamma;
  double Sv[SE_MAXN1 * SE_MAXN1];
  double Tv[SE_MAXN1 * SE_MAXN1];
};

// Device-side error bits (a single unsigned word per library instance).
enum : unsigned {
  KERR_DOMAIN = 1u,            // departure point outside the mesh after the wrap
  KERR_BARRIER_TIMEOUT = 2u,   // a grid barrier wait gave up
  KERR_BAD_CONFIG = 4u,
};

// ---- exact-rounding arithmetic: the reference's coordinate operations, one
// IEEE operation at a time, never contracted into FMAs.
__device__ __forceinline__ double xadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double xsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double xmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double xdiv(double a, double b) { return __ddiv_rn(a, b); }

// ---- double-double arithmetic (error-free transformations: Knuth's TwoSum;
// TwoProd with an FMA): a pair (hi, lo) carries a value to about twice double
// precision. The _rn intrinsics keep each operation one IEEE operation (the
// compiler must not fuse a product into a following sum here).
__device__ __forceinline__ void two_sum(double a, double b, double& s, double& e) {
  s = __dadd_rn(a, b);
  const double bb = __dsub_rn(s, a);
  e = __dadd_rn(__dsub_rn(a, __dsub_rn(s, bb)), __dsub_rn(b, bb));
}
__device__ __forceinline__ void dd_add(double& hi, double& lo, double x) {
  double s, e;
  two_sum(hi, x, s, e);
  hi = s;
  lo += e;
}
__device__ __forceinline__ void dd_fma(double& hi, double& lo, double a, double b) {
  const double p = __dmul_rn(a, b);
  const double pe = fma(a, b, -p);  // exact: a*b - p
  dd_add(hi, lo, p);
  lo += pe;
}

// ---------------------------------------------------------------------------
// Host launch wrappers (defined in sl.cu / linsys.cu). All take the stream.

// SL advection. field: [Nv][ndofs]; vel/vel_prev: [Nv][2]; out: [Nv][ndofs].
// field_prev == nullptr selects the first-order scheme. dep_el/dep_xy are
// optional recordings of the departure elements/points (all vertices).
cudaError_t launch_sl(const MeshDev& m, int ndofs, const double* field, const double* vel,
                      const double* field_prev, const double* vel_prev, double dt,
                      double* out, int* dep_el, double* dep_xy, unsigned* err,
                      cudaStream_t s);
// Mesh::GlobalToLocal at points (device arrays).
cudaError_t launch_global_to_local(const MeshDev& m, const double* pts, int npts, int* el,
                                   double* lc, cudaStream_t s);
// Field::InterpGlobal at points (device arrays).
cudaError_t launch_interp_global(const MeshDev& m, int ndofs, const double* vals,
                                 const double* pts, int npts, double* out, cudaStream_t s);
// NavierStokesEqn pressure step (sl.cu): kind 0 out = div(a) (a 2
// components), kind 2 out = div(a) * 1.5 * 10.0, kind 1 out = a - dt grad p;
// derivatives as InterpDerivsGlobal at the vertices. err (may be null) gets
// KERR_BAD_CONFIG if a vertex does not snap to an element's nodes.
cudaError_t launch_ns_pressure(const MeshDev& m, int kind, const double* a, const double* p,
                               double dt, double* out, unsigned* err, cudaStream_t s);
// Component dof of a 2-component field to (to_scalar) or from a scalar field.
cudaError_t launch_component(int nv, int to_scalar, int dof, double* two, double* one,
                             cudaStream_t s);
// Two-layer QG step pieces (sl.cu): GenPV; pointwise combinations (kind 0
// Helmholtz rhs, 1 Poisson rhs, 2 stream functions and vorticities); SolveQ
// with the dissipation rhs over the unknowns of (dx, dy). grad is
// vel-layout (-d/dy, d/dx) of omegaHat from launch_gen_vel.
cudaError_t launch_gen_pv(const MeshDev& m, const double* omega, const double* psi_i,
                          const double* psi_j, double F, double beta, double* alpha, cudaStream_t s);
cudaError_t launch_qg_combine(const MeshDev& m, int kind, const double* a, const double* b,
                              const double* t, const double* c, double F1, double F2, double cb,
                              double* out0, double* out1, double* out2, double* out3,
                              cudaStream_t s);
cudaError_t launch_qg_solve_q(const MeshDev& m, const Dir& dx, const Dir& dy, double dt,
                              const double* q, const double* tau, const double* omh,
                              const double* grad, const double* tau_e, double rF, double Ei,
                              double nu, double a, double* alpha, cudaStream_t s);
// vel[Nv][2] = (-d psi/dy, d psi/dx) at every vertex (GenVel of SE's QG models).
cudaError_t launch_gen_vel(const MeshDev& m, const double* psi, double* vel, unsigned* err,
                           cudaStream_t s);
// Field::PeriodicUpdate.
cudaError_t launch_periodic_update(const MeshDev& m, int ndofs, double* vals, cudaStream_t s);
// Quadrature sums over all elements: sum detJ*w*a (Integrate) or, with
// b != nullptr, sums of detJ*w*(a-b)^2 and detJ*w*b^2 (FieldError).
// Results land in out2[0..1] (device), deterministic order.
cudaError_t launch_quadrature(const MeshDev& m, int ndofs, int dof, const double* a,
                              const double* b, double* scratch, int nscratch, double* out2,
                              cudaStream_t s);
// Max over vertices of |v|^2 (CalcTimeStep), deterministic.
cudaError_t launch_max_speed_sq(int nv, const double* vel, double* scratch, int nscratch,
                                double* out, cudaStream_t s);

// Linear-system pieces.
// y = A x, element-structured (apply.cu); the reduced-precision form reads
// x in FP16 (fp16 != 0) or BF16 and computes and writes FP32.
// err (nullable): device error word for KERR_BARRIER_TIMEOUT.
cudaError_t launch_op_apply(const OpDev& op, const double* x, double* y, unsigned* err,
                            cudaStream_t s);
cudaError_t launch_op_apply_low(const OpDev& op, int fp16, const void* x, float* y, cudaStream_t s);
// r = b - A x with per-block partial sums (partial[2*block]: (w r)^2 or, when
// natural, r w r; and r^2) over residual_blocks(op) blocks (cg.cu).
cudaError_t launch_residual(const OpDev& op, const double* x, const double* b, double* r,
                            const double* w, int natural, double* partial, cudaStream_t s);
// The same residual with the FDM refinement loop's tail fused in: the block
// that finishes last (arrival counter *count, zero between launches) sums
// the partials in block order into res[0..1], runs the convergence test on
// the loop state and sets the loop's while-condition h.
// split_hi/split_lo (nullable): also write r's TF32 hi/lo split, rows of
// split_pitch FP32 (the tensor-core inverse's input).
struct FdmParams;
struct FdmState;
struct ResTail {
  double* res;
  unsigned* count;
  const FdmParams* p;
  FdmState* st;
  cudaGraphConditionalHandle h;
};
cudaError_t launch_residual_check(const OpDev& op, const double* x, const double* b, double* r,
                                  const double* w, int natural, double* partial, double* res,
                                  unsigned* count, const FdmParams* p, FdmState* st,
                                  cudaGraphConditionalHandle h, cudaStream_t s,
                                  float* split_hi = nullptr, float* split_lo = nullptr,
                                  int split_pitch = 0);
// The element-factored residual of orders 4 to 8 without an SVV term
// (apply.cu); false when the operator needs the general kernel.
bool residual_ef_supported(const OpDev& op);
// Partial-sum pairs launch_residual (with b and partial given) writes.
int residual_partial_blocks(const OpDev& op);
cudaError_t launch_residual_ef(const OpDev& op, const double* x, const double* b, double* r,
                               const double* w, int natural, double* partial, const ResTail& tail,
                               float* split_hi, float* split_lo, int split_pitch, cudaStream_t s);
int residual_blocks(const OpDev& op);
cudaError_t launch_op_diag(const OpDev& op, double* d, cudaStream_t s);
// f = Mass*rhs over the unknowns (FieldRHS + Vector::Assemble), plus lift.
cudaError_t launch_rhs_assemble(const OpDev& op, const MeshDev& m, const double* rhs_vals,
                                const double* lift, double* f, cudaStream_t s);
// lift = -A[unknowns, Dirichlet] * sol_vals[Dirichlet].
cudaError_t launch_lift(const OpDev& op, const MeshDev& m, const double* sol_vals, double* lift,
                        cudaStream_t s);
// dst[0, n) = src[0, n) on the stream (device arrays that do not overlap).
cudaError_t launch_copy(double* dst, const double* src, size_t n, cudaStream_t s);
// sol_vals[unknown vertices and their periodic copies] = x; with st and
// st_host (the device address of a mapped page-locked buffer) also
// *st_host = *st.
cudaError_t launch_update_field(const OpDev& op, const MeshDev& m, const double* x,
                                double* sol_vals, cudaStream_t s, const FdmState* st = nullptr,
                                FdmState* st_host = nullptr);

// Persistent CG over a batch of solves.
struct CgSolve {
  OpDev op;
  const double* b;  // right-hand side (unknowns)
  double *x, *r, *z, *p0, *p1, *w;
  double* dinv;     // Jacobi inverse (streaming mode only)
  double rtol, atol, dtol;
  int max_it;
  int norm_type;
  int remove_null;
  int n;  // unknowns
  // segment range of this solve in the partial-sum table
  int seg_begin, seg_end;
  // state (written by the kernel)
  double beta, betaold, dpi, dpiold, rnorm0, ttol, dp, bcoef, a, zmean;
  int its, reason, done, pbuf;
};
struct CgTile {
  int solve;
  int x0, y0;  // first unknown column/row of the tile
  int seg;     // partial-sum segment this tile accumulates into
};
struct CgBatch {
  CgSolve* solves;  // device array
  int nsolves;
  const CgTile* tiles;  // device array, grouped by block (contiguous chunks)
  const int* block_tile_begin;  // [grid+1]
  double* partials;  // [2][nseg][4]: double-buffered by pass parity
  int nseg;
  unsigned* bar_count;
  unsigned* bar_gen;
  int* n_active;
  unsigned* err;
};
constexpr int kCgTileX = 32;
constexpr int kCgTileY = 16;
constexpr int kCgThreads = kCgTileX * kCgTileY;
// Shared memory of the standalone operator apply for order maxN.
size_t cg_smem_bytes(int maxN);
// Tiles a block may own in the register-resident CG mode.
constexpr int kCgResidentTiles = 4;
// Dynamic shared memory of one CG block (order N, nsolves per launch).
size_t cg_dyn_smem_bytes(int N, int nsolves);
// Blocks of kCgThreads that can be co-resident for the CG kernel.
int cg_max_grid(int device, int N, bool resident, int nsolves, int lowp = 0);
// Persistent CG over a batch of same-order solves; resident needs every block
// to own at most kCgResidentTiles tiles.
// lowp: 0 the FP64 apply; 1 (BF16) or 2 (FP16): the CG's direction vector
// rounded to that type for the operator apply, computed in FP32 (orders 4 to
// 8, no SVV term); dots, updates and the other vectors stay FP64.
cudaError_t launch_cg(const CgBatch& batch, int grid, int N, bool resident, cudaStream_t s,
                      int lowp = 0);

// Device-resident parameters and state of an FDM refinement loop.
struct FdmParams {
  double rtol, atol, dtol;
  int max_it, pad;
};
struct FdmState {
  double rnorm0, ttol, dp, best;
  int its, reason, stalled;
  unsigned kerr;  // KERR_* bits of the loop's kernels (zeroed by the loop's set-up)
};
// Set up the loop from res = {norm^2 of f, .}: rnorm0, tolerance, the
// iteration-0 test; sets the while-condition (1 = iterate).
cudaError_t launch_fdm_init(const FdmParams* p, FdmState* st, const double* res,
                            cudaGraphConditionalHandle h, cudaStream_t s);
// The prologue of an FDM solve in one launch (linsys.cu): f as
// launch_rhs_assemble, r = f, x = 0, res = {norm^2 of f (weights w, natural
// or not), |f|^2} and the loop's set-up as launch_fdm_init. partial holds at
// least 2 * npart doubles; count is zero on entry and on return.
cudaError_t launch_fdm_prologue(const OpDev& op, const MeshDev& m, const double* rhs_vals,
                                const double* lift, double* f, double* r, double* x,
                                const double* w, int natural, double* partial, int npart,
                                double* res, unsigned* count, const FdmParams* p, FdmState* st,
                                cudaGraphConditionalHandle h, cudaStream_t s);
// After a refinement step: iteration count, the residual tests (RTOL, ATOL,
// DTOL, NANORINF, ITS, and stagnation at the rounding floor) and the
// while-condition.
cudaError_t launch_fdm_check(const FdmParams* p, FdmState* st, const double* res,
                             cudaGraphConditionalHandle h, cudaStream_t s);

// FDM products on the tcgen05 tensor cores (tc_gemm.cu): D (M x N) = A B with
// A = (a_hi + a_lo) stored [M][K] (pitch a_pitch) and B stored transposed as
// (b_hi + b_lo) [N][K] (pitch b_pitch), FP32 pairs whose hi parts are TF32
// numbers; three kind::tf32 MMAs per K step (Ah Bh + Ah Bl + Al Bh). Element
// (m, n) of D goes to [n * pitch + m]: kind TC_EPI_SPLIT stores the hi/lo
// split of D, TC_EPI_DIVIDE that of D / (alpha + bm lm[m] + bn ln[n]) (0 where
// the divisor is at most null_tol in magnitude), TC_EPI_ACC64 adds D to an
// FP64 array. Pitches are multiples of 4; bases 16-byte aligned; err must be
// set (KERR_BARRIER_TIMEOUT when a bounded wait gave up).
enum { TC_EPI_SPLIT = 0, TC_EPI_DIVIDE = 1, TC_EPI_ACC64 = 2 };
struct TcEpi {
  int M, N, K;
  float *out_hi, *out_lo;  // SPLIT / DIVIDE: the next product's operand pair
  int pitch;
  double* out64;           // ACC64
  const double *lm, *ln;   // DIVIDE
  double alpha, bm, bn, null_tol;
  unsigned* err;
};
// A product planned once per buffer set (tile shape, tensor maps), launched
// as often as needed.
struct TcPlan {
  CUtensorMap maps[4];
  TcEpi e;
  int epi, bn, ck;
};
cudaError_t tc_plan(TcPlan* p, int epi, const float* a_hi, const float* a_lo, int a_pitch,
                    const float* b_hi, const float* b_lo, int b_pitch, const TcEpi& e);
cudaError_t launch_tc_plan(const TcPlan& p, cudaStream_t s);
// hi/lo split of an FP64 [rows][cols] array (leading dimension ld) into FP32
// arrays of the given pitch: hi = x rounded to TF32, lo = x - hi in FP32.
cudaError_t launch_tc_split(const double* x, int rows, int cols, int ld, float* hi, float* lo,
                            int pitch, cudaStream_t s);

// C = A B (row-major, leading dimensions lda/ldb/ldc) on the tensor cores
// (gemm.cu). prec: 0 FP64, 1 TF32 on FP32 data, 2 BF16. epi: 0 store,
// 1 store after the spectral divide by alpha + bx lx[col] + by ly[row]
// (|divisor| <= null_tol gives 0), 2 accumulate into FP64 C scaled by *cmax
// (cmax == nullptr: 1). a_fp64: A is FP64 (scaled by 1/*amax when amax is
// given) whatever prec; c_fp64: C is FP64 (required for epi 2).
//
// low (FP64 only, k in 1..8): the lowest k x k block of spectral coefficients
// carried apart from the backward transform. With epi 1 the block of C
// (rows and columns < k) is moved into zlow[k][k] and left 0 in C; with
// epi 0 or 2 the product's outputs get sum_a A[r][a] U[a][c] added, U[a][c] =
// sum_b zlow[a][b] ex[c * ldex + b], in double-double (with the old value
// for epi 2), rounded once.
// One periodic direction of nel = 2^logn equal elements of order p in Bloch
// form (bloch.cu): V [nel][p][p] complex, row i column k, the W-orthonormal
// eigenvectors of wavenumber m; mu [nel][p] their eigenvalues; tw [nel/2]
// the FFT twiddles exp(-2 pi i j / nel).
struct BlochDir {
  int nel, p, logn;
  const double2* V;
  const double* mu;
  const double2* tw;
};
// x (= or +=) A^{-1} in for a doubly periodic system by Bloch waves (three
// launches); xh: bloch_spectrum_elems complex work. Shared memory limits:
// 16 p nel bytes (x direction) and 32 p nel bytes (y) each at most 48 KB.
// gate (nullable): a refinement loop's state; when its reason is set on
// the device, in is read as zero (the step adds nothing).
cudaError_t launch_bloch_inverse(const BlochDir& bx, const BlochDir& by, double alpha, double cx,
                                 double cy, double null_tol, const double* in, double* out,
                                 bool accumulate, double2* xh, const FdmState* gate,
                                 cudaStream_t s);
size_t bloch_spectrum_elems(const BlochDir& bx, const BlochDir& by);

struct FdmLow {
  double* zlow;
  const double* ex;
  int ldex, k;
};
cudaError_t launch_fdm_gemm(int prec, int epi, const void* A, int a_fp64, const void* B, void* C,
                            int c_fp64, int M, int N, int K, int lda, int ldb, int ldc,
                            const double* amax, const double* cmax, const double* lx,
                            const double* ly, double alpha, double bx, double by, double null_tol,
                            cudaStream_t s, const FdmLow* low = nullptr,
                            const int* gate = nullptr);

// Fast-diagonalization pieces (fdm.cu). prec: 0 FP64, 1 FP32, 2 BF16.
cudaError_t launch_spectral_divide(int prec, void* v, int gx, int gy, const double* lx,
                                   const double* ly, double alpha, double bx, double by,
                                   double null_tol, cudaStream_t s);
// y = x / max (max read from device memory; 0 leaves y = 0).
cudaError_t launch_to_low(int prec, const double* x, void* y, size_t n, const double* max,
                          cudaStream_t s);
// x += y * max.
cudaError_t launch_add_low(int prec, double* x, const void* y, size_t n, const double* max,
                           cudaStream_t s);
// out2 = {sum (w r)^2 or, natural != 0, sum r w r; sum r^2} (w == nullptr:
// w = 1), deterministic.
cudaError_t launch_norms(const double* r, const double* w, size_t n, int natural, double* partial,
                         int npart, double* out2, cudaStream_t s);
// Sum np pairs of partials into out2 (deterministic order).
cudaError_t launch_norm_final(const double* partial, int np, double* out2, cudaStream_t s);
cudaError_t launch_maxabs(const double* x, size_t n, double* partial, int npart, double* out,
                          cudaStream_t s);
cudaError_t launch_sub(const double* b, const double* y, double* r, size_t n, cudaStream_t s);
cudaError_t launch_invert(double* x, size_t n, cudaStream_t s);
// C = A^T (Bh + Bl) in double-double for n x n row-major matrices, returned
// as Ch + Cl (Bl may be null); set-up only.
cudaError_t launch_dd_gemm_tn(int n, const double* A, const double* Bh, const double* Bl,
                              double* Ch, double* Cl, cudaStream_t s);
// y = a y + b x (a == 0: y = b x, y not read)
cudaError_t launch_axpby(double* y, double a, double b, const double* x, size_t n,
                         cudaStream_t s);
// f -= (sum f / sum d) d with d = 1 / dinv: the right-hand side that Jacobi
// CG with the constant null space projected out of every preconditioned
// residual converges to (its limit solves A x = f - c d, c = sum f / sum d).
cudaError_t launch_project_null(double* f, const double* dinv, size_t n, double* partial,
                                int npart, double* sum2, cudaStream_t s);
cudaError_t launch_remove_mean(double* x, size_t n, double* partial, int npart, double* sum2,
                               cudaStream_t s);

}  // namespace seg
