// Host side of the segpu C-ABI (include/segpu.h): object lifetimes, the
// mesh/GLL/boundary tables, device memory and kernel launches.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cusolverDn.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <functional>
#include <mutex>
#include <tuple>
#include <string>
#include <vector>

#include "../../include/segpu.h"
#include "common.cuh"

using namespace seg;

// ------------------------------------------------------------- errors -----
namespace {
thread_local std::string g_err;
thread_local cudaStream_t g_stream = nullptr;  // the calling thread's stream
std::mutex g_scratch_mu;
double* g_scratch = nullptr;  // reductions: partials + results
constexpr int kScratch = 8192;

int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}
int cuda_fail(cudaError_t e, const char* what) {
  return fail(SE_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}
#define CK(call)                                     \
  do {                                               \
    cudaError_t e_ = (call);                         \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
  } while (0)

int ensure_globals() {
  if (g_scratch) return SE_OK;
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) return fail(SE_ERR_CUDA, "no CUDA device available");
  CK(cudaMalloc(&g_scratch, sizeof(double) * (kScratch + 8)));
  return SE_OK;
}

template <class T>
int dalloc(T** p, size_t n) {
  if (n == 0) n = 1;
  cudaError_t e = cudaMalloc((void**)p, n * sizeof(T));
  if (e != cudaSuccess) {
    *p = nullptr;
    cudaGetLastError();
    return fail(e == cudaErrorMemoryAllocation ? SE_ERR_OOM : SE_ERR_CUDA, "cudaMalloc(%zu): %s",
                n * sizeof(T), cudaGetErrorString(e));
  }
  return SE_OK;
}
template <class T>
void dfree(T*& p) {
  if (p) cudaFree(p);
  p = nullptr;
}

// ------------------------------------------------------------ GLL tables --
// GLL nodes, weights and the cardinal-derivative matrix computed by the same
// procedure as the reference's Legendre element (src/base/Legendre.cpp:15-95,
// src/base/Jacobi.cpp:34-89, src/base/Element.cpp:54-106): the Legendre
// polynomial P_N as monomial coefficients from the three-term recurrence,
// evaluated by pow() over terms of matching parity, interior nodes by Newton
// on P_N' from the left in steps of 1e-3, then mirrored and sorted. Keeping the
// procedure keeps the nodes, and so the mesh vertex coordinates, identical to
// the reference's bit for bit.
struct Poly {
  int n;
  double c[SE_MAXN + 3];
};
void poly_next(Poly& out, int n, const Poly& m1, const Poly& m2) {
  out.n = n;
  std::fill(out.c, out.c + SE_MAXN + 3, 0.0);
  const double a = 0.0;
  double c1 = 2 * n * (2 * a + n) * (2 * a + 2 * n - 2);
  double c2 = (2 * a + 2 * n - 1) * (2 * a + 2 * n) * (2 * a + 2 * n - 2);
  double c3 = 2 * (a + n - 1) * (a + n - 1) * (2 * a + 2 * n);
  c2 /= c1;
  c3 /= c1;
  for (int i = 0; i <= m1.n; i++) out.c[i + 1] += c2 * m1.c[i];
  for (int i = 0; i <= m2.n; i++) out.c[i] -= c3 * m2.c[i];
}
double peval(const Poly& p, double x) {
  double s = 0.0;
  for (int i = p.n; i >= 0; i -= 2) s += p.c[i] * std::pow(x, i);
  return s;
}
double pderiv(const Poly& p, double x) {
  double s = 0.0;
  for (int i = p.n; i >= 1; i -= 2) s += p.c[i] * i * std::pow(x, i - 1);
  return s;
}
double pderiv2(const Poly& p, double x) {
  double s = 0.0;
  for (int i = p.n; i >= 2; i -= 2) s += p.c[i] * i * (i - 1) * std::pow(x, i - 2);
  return s;
}

struct Gll {
  int N;
  double x[SE_MAXN1], w[SE_MAXN1], dC[SE_MAXN1 * SE_MAXN1], lambda[SE_MAXN1];
  double Kh[SE_MAXN1 * SE_MAXN1];
};
void gll_build(int N, Gll& g) {
  g.N = N;
  Poly P[SE_MAXN + 3];
  P[0].n = 0;
  std::fill(P[0].c, P[0].c + SE_MAXN + 3, 0.0);
  P[0].c[0] = 1.0;
  P[1].n = 1;
  std::fill(P[1].c, P[1].c + SE_MAXN + 3, 0.0);
  P[1].c[1] = 1.0;
  for (int i = 2; i <= N + 1; i++) poly_next(P[i], i, P[i - 1], P[i - 2]);
  const Poly& PN = P[N];
  double* x = g.x;
  x[0] = -1.0;
  const double step = 1.0e-3;
  const int half = ((N + 1) % 2 == 1) ? N / 2 : (N + 1) / 2;
  for (int i = 1; i < half; i++) {
    double x0 = x[i - 1];
    bool again;
    do {
      x0 += step;
      double r = x0, rp;
      for (int it = 0; it < 100000; it++) {
        rp = r;
        r = rp - pderiv(PN, rp) / pderiv2(PN, rp);
        if (std::fabs(r - rp) < 1.0e-12) break;
      }
      x[i] = r;
      again = r > 0.0 - step;
      for (int k = 0; k < i && !again; k++)
        if (std::fabs(x[k] - r) < 1.0e-6) again = true;
    } while (again);
    x[N - i] = -x[i];
  }
  x[N] = 1.0;
  if ((N + 1) % 2 == 1) x[(N + 1) / 2] = 0.0;
  // ascending selection sort (ties keep the first occurrence)
  {
    double tmp[SE_MAXN1];
    bool done[SE_MAXN1] = {false};
    int mi = 0;
    for (int i = 0; i <= N; i++) {
      double mv = 1.0e+99;
      for (int j = 0; j <= N; j++)
        if (!done[j] && x[j] < mv) {
          mv = x[j];
          mi = j;
        }
      tmp[i] = mv;
      done[mi] = true;
    }
    std::copy(tmp, tmp + N + 1, x);
  }
  g.w[0] = 2.0 / ((N + 1) * N);
  for (int i = 1; i < N; i++) g.w[i] = 2.0 / ((N + 1) * N * peval(PN, x[i]) * peval(PN, x[i]));
  g.w[N] = 2.0 / ((N + 1) * N);
  Poly PP;
  poly_next(PP, N, P[N - 1], P[N - 2]);
  for (int i = 0; i <= N; i++)
    for (int j = 0; j <= N; j++) {
      double v;
      if (i == j && i == 0)
        v = -0.25 * N * (N + 1);
      else if (i == j && i == N)
        v = +0.25 * N * (N + 1);
      else if (i == j)
        v = 0.0;
      else
        v = peval(PP, x[i]) / (peval(PP, x[j]) * (x[i] - x[j]));
      g.dC[i * (N + 1) + j] = v;
    }
  // Lagrange product weights and the 1-D stiffness Kh = D^T diag(w) D, in
  // extended precision from the double tables.
  for (int j = 0; j <= N; j++) {
    long double p = 1.0L;
    for (int k = 0; k <= N; k++)
      if (k != j) p *= (long double)x[j] - (long double)x[k];
    g.lambda[j] = (double)(1.0L / p);
  }
  for (int a = 0; a <= N; a++)
    for (int b = 0; b <= N; b++) {
      long double s = 0.0L;
      for (int q = 0; q <= N; q++)
        s += (long double)g.w[q] * (long double)g.dC[q * (N + 1) + a] *
             (long double)g.dC[q * (N + 1) + b];
      g.Kh[a * (N + 1) + b] = (double)s;
    }
}
}  // namespace

// ------------------------------------------------------------- objects ----
struct se_mesh {
  Gll gll;
  MeshDev dev;
  int nVertsTotal;
};
struct se_bcs {
  se_mesh* mesh;
  int bottom, top, left, right;  // after the periodic adjustments
  Dir d[2];                      // unknown ranges (operator fields filled later)
  int vec_size;
};
struct se_field {
  se_mesh* mesh;
  int ndofs;
  se_bcs* bcs;
  double* vals;  // device [nVertsTotal][ndofs]
};
struct se_advector {
  se_field *field, *vel, *field_prev, *vel_prev;
  se_field* sl;
  int* dep_el;
  double* dep_xy;
  unsigned* err;  // device error bits of this advector's SL kernels
  bool record;
};
struct se_linsys {
  se_field *sol, *rhs;
  bool poisson;
  double c, nu, dt;
  int svv;  // svvCutoff of a HelmholtzEqn with the SVV operator (0: none)
  se_solver_opts opts;
  se_bcs* own_bcs;  // when sol has no BCs: natural boundaries, all vertices unknown
  OpDev op;
  int n;
  bool assembled;
  double *f, *lift, *x, *r, *z, *p0, *p1, *w, *dinv;
  bool resident;
  // single-solve CG schedule
  CgSolve* d_solve;
  CgTile* d_tiles;
  int* d_block_begin;
  double* d_partials;
  unsigned* d_bar;  // [0] arrivals, [1] generation
  int* d_active;
  unsigned* d_err;
  int grid, nseg, seg_begin, seg_end;
  cudaEvent_t ev[3];  // FDM solve: graph start, graph end, state copied to the host
  // fast diagonalization (built on the first FDM solve)
  bool fdm_ready;
  int fdm_prec;
  // eigenvectors E per direction (W-orthonormal; cached, shared): S = row-major
  // E^T, ST = row-major E; eigenvalues lx, ly
  double *Sx, *Sy, *SxT, *SyT, *lx, *ly;
  void *Sx_lo, *Sy_lo, *SxT_lo, *SyT_lo;  // low-precision copies (cached, shared)
  int fdm_lbuf_prec;          // precision the L2, L3 buffers were sized for
  double *X1, *X2, *ax;       // FP64 work: two transform buffers, A x
  double* zlow;               // FP64 inverse: the low spectral block [lowk][lowk]
  int lowk;
  // FP64 inverse of a doubly periodic system with 2^k elements per
  // direction: Bloch form (bloch.cu) with its complex spectral work array
  bool bloch;
  BlochDir bdx, bdy;
  double2* xh;
  // CG with the reduced-precision apply in FP64 refinement: outer residual,
  // inner solution, norm partials [2 * mx_np] + results [16]
  double *mx_r, *mx_d, *mx_part;
  int mx_np;
  void *L1, *L2, *L3;         // low-precision work (L1 unused)
  // tcgen05 path (SE_PREC_MIXED): operand pairs of the eigenvector products
  // (cached per direction) and two work pairs, [G_y][tc_px] and [G_x][tc_py]
  const float *tcSx[2], *tcSy[2], *tcSxT[2], *tcSyT[2];
  float *tcY[2], *tcX[2];
  int tc_px, tc_py, tc_sms;
  TcPlan* tc_plan;  // the four products' plans (for the output tc_out)
  double* tc_out;
  double* fpart;              // reduction partials [2*fpart_n] + results [16]
  int fpart_n;
  double lmax[2];  // largest 1-D eigenvalue magnitude per direction
  cudaGraphExec_t fdm_exec;  // the captured FDM solve
  int fdm_key;
  FdmParams* d_fparams;
  FdmState* d_fstate;
  unsigned* d_rescount;  // arrival counter of the fused residual + test (zero between launches)
  FdmParams* h_fparams;  // pinned host copies for asynchronous transfers
  FdmState* h_fstate;
  // device address of h_fstate when the pinned buffer is mapped (the solve
  // graph's last kernel then writes the state there), else null
  FdmState* h_fstate_dev;
  bool fdm_state_mapped;  // the current solve graph writes h_fstate_dev
  FdmParams fparams_last;    // the parameters in d_fparams
  bool fparams_sent;         // d_fparams holds fparams_last
  int async_pending;       // 1: FDM solve queued; 2: synchronous result held
  int async_rc;
  se_solve_stats async_stats;
};

namespace {
// Unknown range along one direction (the rectangle the reference's BCs maps
// select: src/base/BCs.cpp:36-195).
Dir make_dir(const MeshDev& m, int d, bool lo_bc, bool hi_bc) {
  Dir r;
  r.nE = m.nEls[d];
  r.N = m.N;
  r.nV = m.nVerts[d];
  r.periodic = m.periodic[d];
  r.lo = lo_bc ? 1 : 0;
  r.hi = (r.periodic || hi_bc) ? r.nV - 1 : r.nV;
  return r;
}

// 1-D factors of SVV(constant, mN)'s element matrix (src/base/SVV.cpp:
// 120-176) on SE's rectangles, where it equals
//     2 constant detJ (T along y (x) S along x),
// S = (F D)^T diag(w) (F D), T = F^T diag(w) F, with F = B diag(q) B^-1 the
// nodal form of the modal filter: B[a][k] the modal basis of
// src/base/Legendre.cpp:307-335 ((1+x)/2, (1-x)/2, (1-x^2)/4 P_{k-2}^(1,1))
// at the GLL node a, q(k) = sqrt(exp(-(N-k)^2/(mN-k)^2)) for k > mN, else
// 0, D the cardinal derivatives. (The reference's Lyy is formed from the x
// derivative again, so both of its terms are this same matrix.) Computed in
// long double.
void svv_factors(const Gll& g, int mN, double* S, double* T) {
  typedef long double L;
  const int N = g.N, n = N + 1;
  // Jacobi P^(1,1) coefficients by the reference's recurrence (src/base/Jacobi.cpp:21-36)
  L P[SE_MAXN1][SE_MAXN1 + 1] = {};
  P[0][0] = 1.0L;
  if (N >= 1) P[1][1] = 2.0L;
  for (int k = 2; k <= N; k++) {
    const L a = 1.0L;
    const L c1 = 2 * k * (2 * a + k) * (2 * a + 2 * k - 2);
    const L c2 = (2 * a + 2 * k - 1) * (2 * a + 2 * k) * (2 * a + 2 * k - 2) / c1;
    const L c3 = 2 * (a + k - 1) * (a + k - 1) * (2 * a + 2 * k) / c1;
    for (int i = 0; i < k; i++) P[k][i + 1] += c2 * P[k - 1][i];
    for (int i = 0; i <= k - 2; i++) P[k][i] -= c3 * P[k - 2][i];
  }
  L modal[SE_MAXN1][SE_MAXN1 + 1] = {};
  modal[0][0] = 0.5L, modal[0][1] = 0.5L;
  modal[1][0] = 0.5L, modal[1][1] = -0.5L;
  for (int k = 2; k <= N; k++)
    for (int j = 0; j < k - 1; j++) {
      modal[k][j] += 0.25L * P[k - 2][j];
      modal[k][j + 2] -= 0.25L * P[k - 2][j];
    }
  L B[SE_MAXN1][SE_MAXN1], Bi[SE_MAXN1][SE_MAXN1], A[SE_MAXN1][SE_MAXN1];
  for (int a = 0; a < n; a++)
    for (int k = 0; k < n; k++) {
      L v = 0.0L;
      for (int i = N; i >= 0; i--) v = v * (L)g.x[a] + modal[k][i];
      B[a][k] = v;
      A[a][k] = v;
      Bi[a][k] = a == k ? 1.0L : 0.0L;
    }
  for (int c = 0; c < n; c++) {  // Gauss-Jordan, partial pivoting
    int p = c;
    for (int r = c + 1; r < n; r++)
      if (fabsl(A[r][c]) > fabsl(A[p][c])) p = r;
    for (int k = 0; k < n; k++) {
      std::swap(A[c][k], A[p][k]);
      std::swap(Bi[c][k], Bi[p][k]);
    }
    const L inv = 1.0L / A[c][c];
    for (int k = 0; k < n; k++) A[c][k] *= inv, Bi[c][k] *= inv;
    for (int r = 0; r < n; r++) {
      if (r == c) continue;
      const L f = A[r][c];
      for (int k = 0; k < n; k++) A[r][k] -= f * A[c][k], Bi[r][k] -= f * Bi[c][k];
    }
  }
  L q[SE_MAXN1], F[SE_MAXN1][SE_MAXN1], FD[SE_MAXN1][SE_MAXN1];
  for (int k = 0; k < n; k++) {
    q[k] = 0.0L;
    if (k > mN) {
      const L e = -((L)(N - k) * (N - k)) / ((L)(mN - k) * (mN - k));
      q[k] = sqrtl(expl(e));
    }
  }
  for (int a = 0; a < n; a++)
    for (int b = 0; b < n; b++) {
      L v = 0.0L;
      for (int k = 0; k < n; k++) v += B[a][k] * q[k] * Bi[k][b];
      F[a][b] = v;
    }
  for (int a = 0; a < n; a++)
    for (int b = 0; b < n; b++) {
      L v = 0.0L;
      for (int c = 0; c < n; c++) v += F[a][c] * (L)g.dC[c * n + b];
      FD[a][b] = v;
    }
  for (int b = 0; b < n; b++)
    for (int c = 0; c < n; c++) {
      L s = 0.0L, t = 0.0L;
      for (int a = 0; a < n; a++) {
        s += FD[a][b] * (L)g.w[a] * FD[a][c];
        t += F[a][b] * (L)g.w[a] * F[a][c];
      }
      S[b * n + c] = (double)s;
      T[b * n + c] = (double)t;
    }
}

void fill_op(se_linsys* ls) {
  const se_mesh* me = ls->sol->mesh;
  const MeshDev& m = me->dev;
  const se_bcs* b = ls->sol->bcs ? ls->sol->bcs : ls->own_bcs;
  OpDev& op = ls->op;
  std::memset(&op, 0, sizeof(op));
  op.d[0] = b->d[0];
  op.d[1] = b->d[1];
  op.G[0] = op.d[0].hi - op.d[0].lo;
  op.G[1] = op.d[1].hi - op.d[1].lo;
  const double hx = m.dx[0], hy = m.dx[1];
  const double s = ls->poisson ? ls->c : ls->nu * ls->dt;
  const double cm = ls->poisson ? 0.0 : ls->c;
  op.alpha = cm * (0.5 * hx) * (0.5 * hy);
  if (ls->opts.mode == SE_MODE_EXACT) {
    op.beta[0] = s * (hy / hx);
    op.beta[1] = s * (hx / hy);
  } else {
    // the reference's Laplacian drops detJ (src/base/Operator.cpp:72)
    op.beta[0] = s * (2.0 / hx) * (2.0 / hx);
    op.beta[1] = s * (2.0 / hy) * (2.0 / hy);
  }
  const int n = m.N + 1;
  for (int a = 0; a < n * n; a++) op.Kh[a] = me->gll.Kh[a];
  for (int a = 0; a < n; a++) op.w[a] = me->gll.w[a];
  if (ls->svv && !ls->poisson) {
    // SVV(dt, svvCutoff) (src/linsys/HelmholtzEqn.cpp:71) with the true
    // Jacobian in either mode (SVV.cpp:132 uses Mesh::DetJac)
    svv_factors(me->gll, ls->svv, op.Sv, op.Tv);
    op.gamma = 2.0 * ls->dt * ((0.5 * hx) * (0.5 * hy));
  }
}

// Static schedule for one cooperative launch over several solves: tiles of
// kCgTileX x kCgTileY unknowns, grouped solve by solve, split into `grid`
// contiguous chunks; a segment is the run of one solve's tiles inside one
// chunk, so each solve's segments are contiguous.
struct Schedule {
  std::vector<CgTile> tiles;
  std::vector<int> block_begin;
  std::vector<int> seg_begin, seg_end;  // per solve
  int nseg = 0;
};
Schedule make_schedule(const std::vector<const OpDev*>& ops, int max_grid) {
  Schedule S;
  for (size_t s = 0; s < ops.size(); s++) {
    const OpDev& op = *ops[s];
    for (int y = 0; y < op.G[1]; y += kCgTileY)
      for (int x = 0; x < op.G[0]; x += kCgTileX) S.tiles.push_back({(int)s, x, y, 0});
  }
  const int nt = (int)S.tiles.size();
  int grid = std::max(1, std::min(max_grid, nt));
  S.block_begin.resize(grid + 1);
  for (int b = 0; b <= grid; b++) S.block_begin[b] = (int)((long)nt * b / grid);
  S.seg_begin.assign(ops.size(), -1);
  S.seg_end.assign(ops.size(), -1);
  int seg = -1;
  for (int b = 0; b < grid; b++) {
    int last = -1;
    for (int t = S.block_begin[b]; t < S.block_begin[b + 1]; t++) {
      if (S.tiles[t].solve != last) {
        ++seg;
        last = S.tiles[t].solve;
        if (S.seg_begin[last] < 0) S.seg_begin[last] = seg;
        S.seg_end[last] = seg + 1;
      }
      S.tiles[t].seg = seg;
    }
  }
  S.nseg = seg + 1;
  return S;
}


}  // namespace

namespace {
CgSolve make_solve(const se_linsys* ls, const double* b, double* x, double rtol, double atol,
                   double dtol, int max_it, int remove_null) {
  CgSolve cs;
  std::memset(&cs, 0, sizeof(cs));
  cs.op = ls->op;
  cs.b = b;
  cs.x = x;
  cs.r = ls->r;
  cs.z = ls->z;
  cs.p0 = ls->p0;
  cs.p1 = ls->p1;
  cs.w = ls->w;
  cs.dinv = ls->dinv;
  cs.rtol = rtol;
  cs.atol = atol;
  cs.dtol = dtol;
  cs.max_it = max_it;
  cs.norm_type = ls->opts.norm_type;
  cs.remove_null = remove_null;
  cs.n = ls->n;
  cs.seg_begin = ls->seg_begin;
  cs.seg_end = ls->seg_end;
  return cs;
}

void linsys_free(se_linsys* ls) {
  dfree(ls->f);
  dfree(ls->lift);
  dfree(ls->x);
  dfree(ls->r);
  dfree(ls->z);
  dfree(ls->p0);
  dfree(ls->p1);
  dfree(ls->w);
  dfree(ls->dinv);
  dfree(ls->d_solve);
  dfree(ls->d_tiles);
  dfree(ls->d_block_begin);
  dfree(ls->d_partials);
  dfree(ls->d_bar);
  dfree(ls->d_active);
  dfree(ls->d_err);
  dfree(ls->d_rescount);
  dfree(ls->X1);
  dfree(ls->X2);
  dfree(ls->ax);
  dfree(ls->zlow);
  dfree(ls->xh);
  dfree(ls->mx_r);
  dfree(ls->mx_d);
  dfree(ls->mx_part);
  if (ls->L1) cudaFree(ls->L1);
  if (ls->L2) cudaFree(ls->L2);
  if (ls->L3) cudaFree(ls->L3);
  for (int k = 0; k < 2; k++) {
    dfree(ls->tcY[k]);
    dfree(ls->tcX[k]);
  }
  delete[] ls->tc_plan;
  dfree(ls->fpart);
  if (ls->fdm_exec) cudaGraphExecDestroy(ls->fdm_exec);
  dfree(ls->d_fparams);
  dfree(ls->d_fstate);
  if (ls->h_fparams) cudaFreeHost(ls->h_fparams);
  for (cudaEvent_t e : ls->ev)
    if (e) cudaEventDestroy(e);
  delete ls->own_bcs;
  delete ls;
}

// Number of CG tiles of an operator's unknown grid.
long cg_tiles(const OpDev& op) {
  return (long)((op.G[0] + kCgTileX - 1) / kCgTileX) * ((op.G[1] + kCgTileY - 1) / kCgTileY);
}

// Grid and mode of the persistent CG for ntiles tiles of order N: resident
// (state in registers) when every block can own at most kCgResidentTiles
// tiles; otherwise streaming with SE_CG_BLOCKS_PER_SM (default 2) blocks per
// SM. Returns the grid (0 on failure).
int cg_plan(int dev, int N, long ntiles, int nsolves, bool* resident) {
  const int maxr = cg_max_grid(dev, N, true, nsolves);
  if (maxr > 0 && ntiles <= (long)maxr * kCgResidentTiles) {
    *resident = true;
    return (int)std::min<long>(maxr, ntiles);
  }
  int maxs = cg_max_grid(dev, N, false, nsolves);
  if (maxs <= 0) return 0;
  int sms = 1, per = 2;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (const char* e = std::getenv("SE_CG_BLOCKS_PER_SM")) per = std::max(1, std::atoi(e));
  *resident = false;
  return (int)std::min<long>(std::min(maxs, sms * per), ntiles);
}

int linsys_alloc(se_linsys* ls) {
  const int n = ls->n;
  int rc;
  if ((rc = dalloc(&ls->f, n)) || (rc = dalloc(&ls->lift, n)) || (rc = dalloc(&ls->x, n)) ||
      (rc = dalloc(&ls->r, n)) || (rc = dalloc(&ls->z, n)) || (rc = dalloc(&ls->p0, n)) ||
      (rc = dalloc(&ls->p1, n)) || (rc = dalloc(&ls->w, n)) || (rc = dalloc(&ls->dinv, n)))
    return rc;
  CK(cudaMemsetAsync(ls->lift, 0, sizeof(double) * n, g_stream));
  int dev = 0;
  CK(cudaGetDevice(&dev));
  const int grid = cg_plan(dev, ls->op.d[0].N, cg_tiles(ls->op), 1, &ls->resident);
  if (grid <= 0) return fail(SE_ERR_CUDA, "cannot size the cooperative CG launch");
  Schedule S = make_schedule({&ls->op}, grid);
  ls->grid = (int)S.block_begin.size() - 1;
  ls->nseg = S.nseg;
  ls->seg_begin = S.seg_begin[0];
  ls->seg_end = S.seg_end[0];
  if ((rc = dalloc(&ls->d_solve, 1)) || (rc = dalloc(&ls->d_tiles, S.tiles.size())) ||
      (rc = dalloc(&ls->d_block_begin, S.block_begin.size())) ||
      (rc = dalloc(&ls->d_partials, (size_t)S.nseg * 8)) || (rc = dalloc(&ls->d_bar, 2)) ||
      (rc = dalloc(&ls->d_active, 1)) || (rc = dalloc(&ls->d_err, 1)))
    return rc;
  // on the caller's stream, finished before the system is handed out: the
  // library's streams are non-blocking, so nothing orders them against the
  // legacy stream
  CK(cudaMemcpyAsync(ls->d_tiles, S.tiles.data(), sizeof(CgTile) * S.tiles.size(),
                     cudaMemcpyHostToDevice, g_stream));
  CK(cudaMemcpyAsync(ls->d_block_begin, S.block_begin.data(), sizeof(int) * S.block_begin.size(),
                     cudaMemcpyHostToDevice, g_stream));
  CK(cudaMemsetAsync(ls->d_bar, 0, 2 * sizeof(unsigned), g_stream));
  CK(cudaMemsetAsync(ls->d_err, 0, sizeof(unsigned), g_stream));
  CK(cudaStreamSynchronize(g_stream));
  return SE_OK;
}

// Run the persistent CG for A x = b on this system's schedule; fills stats.
int run_cg(se_linsys* ls, const double* b, double* x, double rtol, double atol, double dtol,
           int max_it, int remove_null, CgSolve* out_state, float* kernel_ms, int lowp = 0) {
  CgSolve cs = make_solve(ls, b, x, rtol, atol, dtol, max_it, remove_null);
  cudaStream_t s = g_stream;
  CK(cudaMemcpyAsync(ls->d_solve, &cs, sizeof(cs), cudaMemcpyHostToDevice, s));
  CK(cudaMemsetAsync(ls->d_bar, 0, sizeof(unsigned), s));  // barrier word starts at 0
  CK(cudaMemsetAsync(ls->d_err, 0, sizeof(unsigned), s));
  CgBatch B;
  B.solves = ls->d_solve;
  B.nsolves = 1;
  B.tiles = ls->d_tiles;
  B.block_tile_begin = ls->d_block_begin;
  B.partials = ls->d_partials;
  B.nseg = ls->nseg;
  B.bar_count = ls->d_bar;
  B.bar_gen = ls->d_bar + 1;
  B.n_active = ls->d_active;
  B.err = ls->d_err;
  if (!ls->ev[0]) {
    CK(cudaEventCreate(&ls->ev[0]));
    CK(cudaEventCreate(&ls->ev[1]));
  }
  CK(cudaEventRecord(ls->ev[0], s));
  CK(launch_cg(B, ls->grid, ls->op.d[0].N, ls->resident, s, lowp));
  CK(cudaEventRecord(ls->ev[1], s));
  unsigned err = 0;
  CK(cudaMemcpyAsync(out_state, ls->d_solve, sizeof(CgSolve), cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(&err, ls->d_err, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  if (kernel_ms) CK(cudaEventElapsedTime(kernel_ms, ls->ev[0], ls->ev[1]));
  if (err & KERR_BARRIER_TIMEOUT) return fail(SE_ERR_TIMEOUT, "CG grid barrier timed out");
  return SE_OK;
}

int check_field(const se_field* f) {
  if (!f || !f->mesh || !f->vals) return fail(SE_ERR_ARG, "null field");
  return SE_OK;
}

// Partial-sum slots of the FDM and refinement norms (at least one per block of
// any norm or residual launch).
constexpr int kFdmPartials = 1184;

// Inner relative tolerance of the reduced-precision CG: each refinement step
// needs only a contraction; tighter inner solves cost more iterations than
// they save in outer steps.
constexpr double kMixedInnerRtol = 1e-2;
constexpr int kMixedMaxOuter = 100;

// SE_METHOD_CG with SE_PREC_BF16 / SE_PREC_FP16: FP64 iterative refinement
// around the persistent CG whose operator apply reads its direction vector
// rounded to BF16 / FP16 and computes in FP32. Every outer step:
//   r = f - A x            (double-double residual, FP64 result)
//   test ||r|| in the chosen norm against max(rtol ||f||, atol)
//   s = RMS of D^-1 r;  solve A d = r / s by that CG to kMixedInnerRtol
//   x += s d               (FP64)
// The dots, updates and vectors of the inner CG stay FP64; the scaling keeps
// FP16 directions inside its range. The apply's rounding perturbs the
// operator by about 2^-9 (BF16) or 2^-12 (FP16) of the direction, so the
// inner solves converge only while that times the system's condition number
// stays well below 1; past it the outer residual stops falling and the solve
// ends with SE_KSP_DIVERGED_BREAKDOWN (the FDM refinement's rule: no 10% gain
// in three steps). out: its = inner CG iterations summed, dp / rnorm0 the
// outer residual norms, reason PETSc's code (2 rtol, 3 atol, -3 iterations,
// -4 dtol, -5 stalled, or the inner CG's breakdown).
int run_mixed_cg(se_linsys* ls, int lowp, CgSolve* out, int* outer, float* kernel_ms) {
  const OpDev& op = ls->op;
  const size_t n = (size_t)ls->n;
  if (op.gamma != 0.0)
    return fail(SE_ERR_UNSUPPORTED, "the reduced-precision CG apply has no SVV term");
  if (op.d[0].N < 4 || op.d[0].N > 8)
    return fail(SE_ERR_UNSUPPORTED, "the reduced-precision CG apply covers orders 4 to 8");
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (ls->grid > cg_max_grid(dev, op.d[0].N, ls->resident, 1, lowp))
    return fail(SE_ERR_UNSUPPORTED, "the reduced-precision CG kernel does not fit the CG grid");
  cudaStream_t s = g_stream;
  if (!ls->mx_r) {
    ls->mx_np = std::max(kFdmPartials, std::max(residual_partial_blocks(op), residual_blocks(op)));
    int rc;
    if ((rc = dalloc(&ls->mx_r, n)) || (rc = dalloc(&ls->mx_d, n)) ||
        (rc = dalloc(&ls->mx_part, 2 * (size_t)ls->mx_np + 16)))
      return rc;
  }
  // Jacobi inverse for the norms (the operator may have changed mode)
  CK(launch_op_diag(op, ls->dinv, s));
  CK(launch_invert(ls->dinv, n, s));
  double* out2 = ls->mx_part + 2 * ls->mx_np;
  const int nt = ls->opts.norm_type;
  // h2[0] = sum (D^-1 r)^2, h2[1] = sum r^2, h2[2] = sum r D^-1 r (natural only)
  double h2[4] = {0.0, 0.0, 0.0, 0.0};
  auto norms = [&](bool fresh_partials) -> int {
    if (fresh_partials)
      CK(launch_norms(ls->mx_r, ls->dinv, n, 0, ls->mx_part, ls->mx_np, out2, s));
    else
      CK(launch_norm_final(ls->mx_part, residual_partial_blocks(op), out2, s));
    CK(cudaMemcpyAsync(h2, out2, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
    if (nt == SE_NORM_NATURAL) {
      CK(launch_norms(ls->mx_r, ls->dinv, n, 1, ls->mx_part, ls->mx_np, out2 + 2, s));
      CK(cudaMemcpyAsync(h2 + 2, out2 + 2, sizeof(double), cudaMemcpyDeviceToHost, s));
    }
    CK(cudaStreamSynchronize(s));
    return SE_OK;
  };
  auto norm = [&]() {
    return std::sqrt(nt == SE_NORM_PRECONDITIONED ? h2[0]
                     : nt == SE_NORM_UNPRECONDITIONED ? h2[1]
                                                      : std::fabs(h2[2]));
  };
  CK(cudaMemsetAsync(ls->x, 0, sizeof(double) * n, s));
  CK(cudaMemcpyAsync(ls->mx_r, ls->f, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
  if (int rc = norms(true)) return rc;
  const double rnorm0 = norm();
  const double ttol = std::max(ls->opts.rtol * rnorm0, ls->opts.atol);
  std::memset(out, 0, sizeof(*out));
  out->rnorm0 = rnorm0;
  float total_ms = 0.f;
  int its = 0, k = 0, reason = 0, stalled = 0;
  double dp = rnorm0, prev = rnorm0;
  for (;; k++) {
    if (dp <= ttol) {
      reason = dp <= ls->opts.atol ? 3 : 2;
      break;
    }
    if (!(dp == dp) || dp > ls->opts.dtol * rnorm0) {
      reason = -4;
      break;
    }
    if (k > 0) {  // the FDM refinement's rule: no 10% gain in three steps
      stalled = dp > 0.9 * prev ? stalled + 1 : 0;
      if (stalled >= 3) {
        reason = SE_KSP_DIVERGED_BREAKDOWN;
        break;
      }
    }
    prev = dp;
    if (its >= ls->opts.max_it || k >= kMixedMaxOuter) {
      reason = -3;
      break;
    }
    const double sc = std::sqrt(h2[0] / (double)n);
    if (!(sc > 0.0)) {
      reason = 2;
      break;
    }
    CK(launch_axpby(ls->mx_r, 0.0, 1.0 / sc, ls->mx_r, n, s));
    CgSolve st;
    float ms = 0.f;
    // an inner solve ends at its tolerance or after n iterations (where CG
    // in exact arithmetic is done; one that stalls on the reduced-precision
    // apply hands the refinement what it has)
    const int inner_max = (int)std::min<long>(ls->opts.max_it - its, std::max<long>(100, (long)n));
    if (int rc = run_cg(ls, ls->mx_r, ls->mx_d, kMixedInnerRtol, 0.0, 1e30, inner_max, 0, &st, &ms,
                        lowp))
      return rc;
    its += st.its;
    total_ms += ms;
    if (st.reason < 0 && st.reason != -3) {  // breakdown or indefinite inner system
      reason = st.reason;
      break;
    }
    CK(launch_axpby(ls->x, 1.0, sc, ls->mx_d, n, s));
    CK(launch_residual(op, ls->x, ls->f, ls->mx_r, ls->dinv, 0, ls->mx_part, s));
    if (int rc = norms(false)) return rc;
    dp = norm();
  }
  out->its = its;
  out->dp = dp;
  out->reason = reason;
  *outer = k;
  if (kernel_ms) *kernel_ms = total_ms;
  return SE_OK;
}
}  // namespace


// ------------------------------------------------- fast diagonalization ----
namespace {
// 1-D assembled stiffness (dense, n x n) and weights on one direction's
// unknowns: element rows of Kh and w added at the vertices they map to
// (periodic end folded onto the start, Dirichlet vertices dropped).
void assemble_1d(const Dir& d, const double* Kh, const double* w, std::vector<double>& K,
                 std::vector<double>& W) {
  const int n = d.hi - d.lo, N = d.N;
  K.assign((size_t)n * n, 0.0);
  W.assign(n, 0.0);
  auto u = [&](int g) {
    if (d.periodic && g == d.nV - 1) g = 0;
    return (g >= d.lo && g < d.hi) ? g - d.lo : -1;
  };
  for (int e = 0; e < d.nE; e++)
    for (int a = 0; a <= N; a++) {
      const int ua = u(e * N + a);
      if (ua < 0) continue;
      W[ua] += w[a];
      for (int b = 0; b <= N; b++) {
        const int ub = u(e * N + b);
        if (ub >= 0) K[(size_t)ua * n + ub] += Kh[a * (N + 1) + b];
      }
    }
}

// Row pitch (in FP32) of a tcgen05 operand with n columns: whole 128-byte
// rows, so that the TMA strides are multiples of 16 bytes.
int tc_pitch(int n) { return (n + 31) / 32 * 32; }
// f rounded to the nearest TF32 number (ties away from zero), as cvt.rna.tf32.
float tf32_rna(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  u = (u + 0x1000u) & 0xFFFFE000u;
  std::memcpy(&f, &u, 4);
  return f;
}

uint16_t to_bf16(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  u += 0x7fffu + ((u >> 16) & 1u);  // round to nearest even
  return (uint16_t)(u >> 16);
}

// Host-to-device copy complete on return (set-up data that kernels on any of
// the library's non-blocking streams read afterwards).
cudaError_t upload_now(void* dst, const void* src, size_t bytes) {
  cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, g_stream);
  return e != cudaSuccess ? e : cudaStreamSynchronize(g_stream);
}

// One step of iterative refinement of generalised eigenpairs (Ogita and
// Aishima, "Iterative refinement for symmetric eigenvalue decomposition",
// Japan J. Indust. Appl. Math. 35, 2018, Algorithm 1, in the W inner
// product): with R = I - E^T W E and S = E^T K E formed in double-double on
// the device, l_i = S_ii / (1 - R_ii) and
//   F_ij = (S_ij + l_j R_ij) / (l_j - l_i)   if |l_j - l_i| > delta,
//   F_ij = R_ij / 2                           otherwise (a cluster),
// E <- E + E F. One step takes syevd's eigenvectors (errors near 1e-13 on
// close pairs) to about the FP64 rounding of the exact ones; this is what
// lets one FP64 refinement step of the fast-diagonalization solve reach
// 1e-10 on smooth right-hand sides. delta = 2 (max|S - diag(l)| +
// max|l| max|R|), at least 1e-10 max|l| (exactly degenerate pairs, such as
// the sine and cosine modes of a periodic direction, stay one cluster).
// E column-major (E[j*n + i] = entry (i, j)); K row-major, symmetric.
int refine_eig(int n, const std::vector<double>& K, const std::vector<double>& W,
               std::vector<double>& E, std::vector<double>& lam) {
  const size_t nn = (size_t)n * n;
  std::vector<double> Er(nn), WEh(nn), WEl(nn);
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) {
      const double e = E[(size_t)j * n + i];
      Er[(size_t)i * n + j] = e;
      WEh[(size_t)i * n + j] = W[i] * e;
      WEl[(size_t)i * n + j] = std::fma(W[i], e, -W[i] * e);
    }
  double* buf = nullptr;
  if (int rc = dalloc(&buf, 10 * nn)) return rc;
  double *dK = buf, *dE = buf + nn, *dEc = buf + 2 * nn, *dWh = buf + 3 * nn, *dWl = buf + 4 * nn;
  double *dKh = buf + 5 * nn, *dKl = buf + 6 * nn, *dSh = buf + 7 * nn, *dSl = buf + 8 * nn,
         *dF = buf + 9 * nn;
  std::vector<double> Sh(nn), Sl(nn), Gh(nn), Gl(nn), F(nn);
  cudaStream_t s = g_stream;
  auto run = [&]() -> cudaError_t {
    cudaError_t e;
    if ((e = cudaMemcpyAsync(dK, K.data(), 8 * nn, cudaMemcpyHostToDevice, s)) ||
        (e = cudaMemcpyAsync(dE, Er.data(), 8 * nn, cudaMemcpyHostToDevice, s)) ||
        (e = cudaMemcpyAsync(dEc, E.data(), 8 * nn, cudaMemcpyHostToDevice, s)) ||
        (e = cudaMemcpyAsync(dWh, WEh.data(), 8 * nn, cudaMemcpyHostToDevice, s)) ||
        (e = cudaMemcpyAsync(dWl, WEl.data(), 8 * nn, cudaMemcpyHostToDevice, s)))
      return e;
    // K E (K symmetric), S = E^T (K E), G = E^T (W E)
    if ((e = launch_dd_gemm_tn(n, dK, dE, nullptr, dKh, dKl, s)) ||
        (e = launch_dd_gemm_tn(n, dE, dKh, dKl, dSh, dSl, s)) ||
        (e = launch_dd_gemm_tn(n, dE, dWh, dWl, dKh, dKl, s)))
      return e;
    if ((e = cudaMemcpyAsync(Sh.data(), dSh, 8 * nn, cudaMemcpyDeviceToHost, s)) ||
        (e = cudaMemcpyAsync(Sl.data(), dSl, 8 * nn, cudaMemcpyDeviceToHost, s)) ||
        (e = cudaMemcpyAsync(Gh.data(), dKh, 8 * nn, cudaMemcpyDeviceToHost, s)) ||
        (e = cudaMemcpyAsync(Gl.data(), dKl, 8 * nn, cudaMemcpyDeviceToHost, s)))
      return e;
    return cudaStreamSynchronize(s);
  };
  cudaError_t ce = run();
  if (ce != cudaSuccess) {
    dfree(buf);
    return fail(SE_ERR_CUDA, "eigenvector refinement: %s", cudaGetErrorString(ce));
  }
  std::vector<double> l(n), R(nn);
  double maxl = 0.0, maxr = 0.0, maxoff = 0.0;
  for (int i = 0; i < n; i++) {
    const long double sii = (long double)Sh[(size_t)i * n + i] + Sl[(size_t)i * n + i];
    const long double gii = (long double)Gh[(size_t)i * n + i] + Gl[(size_t)i * n + i];
    l[i] = (double)(sii / gii);
    maxl = std::max(maxl, std::fabs(l[i]));
  }
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) {
      const size_t k = (size_t)i * n + j;
      R[k] = ((i == j ? 1.0 : 0.0) - Gh[k]) - Gl[k];
      maxr = std::max(maxr, std::fabs(R[k]));
      const double sij = Sh[k] + Sl[k];
      maxoff = std::max(maxoff, std::fabs(i == j ? sij - l[i] : sij));
    }
  const double delta = std::max(2.0 * (maxoff + maxl * maxr), 1e-10 * maxl);
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) {
      const size_t k = (size_t)i * n + j;
      const double gap = l[j] - l[i];
      F[k] = std::fabs(gap) > delta ? (Sh[k] + Sl[k] + l[j] * R[k]) / gap : 0.5 * R[k];
    }
  // E F = (E^T)^T F, E^T row-major being E column-major
  auto run2 = [&]() -> cudaError_t {
    cudaError_t e;
    if ((e = cudaMemcpyAsync(dF, F.data(), 8 * nn, cudaMemcpyHostToDevice, s)) ||
        (e = launch_dd_gemm_tn(n, dEc, dF, nullptr, dSh, dSl, s)) ||
        (e = cudaMemcpyAsync(Sh.data(), dSh, 8 * nn, cudaMemcpyDeviceToHost, s)) ||
        (e = cudaMemcpyAsync(Sl.data(), dSl, 8 * nn, cudaMemcpyDeviceToHost, s)))
      return e;
    return cudaStreamSynchronize(s);
  };
  ce = run2();
  dfree(buf);
  if (ce != cudaSuccess) return fail(SE_ERR_CUDA, "eigenvector refinement: %s", cudaGetErrorString(ce));
  // Sh + Sl = (E F)[i][j] row-major; E is column-major
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) {
      const size_t k = (size_t)i * n + j;
      E[(size_t)j * n + i] += Sh[k] + Sl[k];
    }
  lam = l;
  return SE_OK;
}

// Generalised eigenvectors S (S^T K S = diag(lam), S^T W S = I) of one
// direction, on the device: eigenvectors of W^-1/2 K W^-1/2 by cuSOLVER
// syevd (setup only), scaled by W^-1/2, then refined (refine_eig).
int eig_1d(const Dir& d, const double* Kh, const double* w, double** S_dev, double** ST_dev,
           double** lam_dev, std::vector<double>& S_host) {
  std::vector<double> K, W;
  assemble_1d(d, Kh, w, K, W);
  const int n = d.hi - d.lo;
  std::vector<double> A((size_t)n * n);
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) A[(size_t)j * n + i] = K[(size_t)i * n + j] / std::sqrt(W[i] * W[j]);
  double *dA = nullptr, *dlam = nullptr, *work = nullptr;
  int* info = nullptr;
  int rc;
  if ((rc = dalloc(&dA, (size_t)n * n)) || (rc = dalloc(&dlam, n)) || (rc = dalloc(&info, 1))) {
    dfree(dA);
    dfree(dlam);
    dfree(info);
    return rc;
  }
  cusolverDnHandle_t h = nullptr;
  int lwork = 0, hinfo = 0;
  bool ok = cusolverDnCreate(&h) == CUSOLVER_STATUS_SUCCESS;
  ok = ok && cudaMemcpy(dA, A.data(), sizeof(double) * A.size(), cudaMemcpyHostToDevice) == cudaSuccess;
  ok = ok && cusolverDnDsyevd_bufferSize(h, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, n, dA, n,
                                         dlam, &lwork) == CUSOLVER_STATUS_SUCCESS;
  ok = ok && dalloc(&work, (size_t)lwork) == SE_OK;
  ok = ok && cusolverDnDsyevd(h, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, n, dA, n, dlam,
                              work, lwork, info) == CUSOLVER_STATUS_SUCCESS;
  ok = ok && cudaMemcpy(&hinfo, info, sizeof(int), cudaMemcpyDeviceToHost) == cudaSuccess && hinfo == 0;
  ok = ok && cudaMemcpy(A.data(), dA, sizeof(double) * A.size(), cudaMemcpyDeviceToHost) == cudaSuccess;
  if (h) cusolverDnDestroy(h);
  dfree(work);
  dfree(info);
  if (!ok) {
    dfree(dA);
    dfree(dlam);
    return fail(SE_ERR_CUDA, "eigendecomposition of the 1-D operator failed (n=%d)", n);
  }
  for (int j = 0; j < n; j++)
    for (int i = 0; i < n; i++) A[(size_t)j * n + i] /= std::sqrt(W[i]);
  {
    std::vector<double> lam(n);
    if (cudaMemcpy(lam.data(), dlam, sizeof(double) * n, cudaMemcpyDeviceToHost) != cudaSuccess) {
      dfree(dA);
      dfree(dlam);
      return fail(SE_ERR_CUDA, "eigenvalue download failed (n=%d)", n);
    }
    if (int rc2 = refine_eig(n, K, W, A, lam)) {
      dfree(dA);
      dfree(dlam);
      return rc2;
    }
    CK(upload_now(dlam, lam.data(), sizeof(double) * n));
  }
  S_host = A;
  CK(upload_now(dA, A.data(), sizeof(double) * A.size()));
  std::vector<double> T((size_t)n * n);
  for (int j = 0; j < n; j++)
    for (int i = 0; i < n; i++) T[(size_t)i * n + j] = A[(size_t)j * n + i];
  double* dT = nullptr;
  if (int rc2 = dalloc(&dT, (size_t)n * n)) {
    dfree(dA);
    dfree(dlam);
    return rc2;
  }
  CK(upload_now(dT, T.data(), sizeof(double) * T.size()));
  *S_dev = dA;
  *ST_dev = dT;
  *lam_dev = dlam;
  return SE_OK;
}

int upload_low(const std::vector<double>& S, int prec, void** out) {
  const size_t n = S.size();
  if (prec == 1) {
    std::vector<float> v(n);
    for (size_t k = 0; k < n; k++) v[k] = (float)S[k];
    float* d = nullptr;
    if (int rc = dalloc(&d, n)) return rc;
    CK(upload_now(d, v.data(), sizeof(float) * n));
    *out = d;
  } else {
    std::vector<uint16_t> v(n);
    for (size_t k = 0; k < n; k++) v[k] = to_bf16((float)S[k]);
    uint16_t* d = nullptr;
    if (int rc = dalloc(&d, n)) return rc;
    CK(upload_now(d, v.data(), sizeof(uint16_t) * n));
    *out = d;
  }
  return SE_OK;
}

// Process-wide cache of 1-D generalised eigendecompositions, per device.
// The 1-D assembled operators depend only on the element count, the order
// and the boundary ends of a direction (not on h, the coefficients or the
// Laplacian scaling), so every system with the same direction shares one
// setup; entries live until the process exits.
struct Eig1D {
  int n = 0;
  double* S = nullptr;    // W-orthonormal eigenvectors E, column-major (= row-major E^T)
  double* ST = nullptr;   // row-major E
  double* lam = nullptr;  // eigenvalues
  double lmax = 0.0;
  void* low[3] = {nullptr, nullptr, nullptr};   // [1] FP32, [2] BF16 copies of S
  void* lowT[3] = {nullptr, nullptr, nullptr};  // and of ST
  // TF32 hi/lo pairs for the tcgen05 products, rows padded to tc_pitch:
  // tc[0] of S (row-major E^T), tc[1] of ST (row-major E); [.][0] hi, [.][1] lo
  float* tc[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
  int tc_pitch = 0;
};
typedef std::tuple<int, int, int, int, int, int> EigKey;
std::mutex g_eig_mu;
std::map<EigKey, Eig1D*> g_eig[64];

int eig_get(const Dir& d, const double* Kh, const double* w, int prec, Eig1D** out) {
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return fail(SE_ERR_UNSUPPORTED, "device index %d", dev);
  std::lock_guard<std::mutex> lk(g_eig_mu);
  const EigKey key(d.nE, d.N, d.periodic, d.lo, d.hi, d.nV);
  Eig1D*& e = g_eig[dev][key];
  std::vector<double> Sh;
  if (!e) {
    Eig1D* ne = new Eig1D();
    ne->n = d.hi - d.lo;
    if (int rc = eig_1d(d, Kh, w, &ne->S, &ne->ST, &ne->lam, Sh)) {
      delete ne;
      g_eig[dev].erase(key);
      return rc;
    }
    std::vector<double> lam(ne->n);
    CK(cudaMemcpy(lam.data(), ne->lam, sizeof(double) * ne->n, cudaMemcpyDeviceToHost));
    for (double v : lam) ne->lmax = std::max(ne->lmax, std::fabs(v));
    e = ne;
  }
  if (prec == 2 && !e->low[prec]) {
    if (Sh.empty()) {
      Sh.resize((size_t)e->n * e->n);
      CK(cudaMemcpy(Sh.data(), e->S, sizeof(double) * Sh.size(), cudaMemcpyDeviceToHost));
    }
    if (int rc = upload_low(Sh, prec, &e->low[prec])) return rc;
    const int n = e->n;
    std::vector<double> T((size_t)n * n);
    for (int j = 0; j < n; j++)
      for (int i = 0; i < n; i++) T[(size_t)i * n + j] = Sh[(size_t)j * n + i];
    if (int rc = upload_low(T, prec, &e->lowT[prec])) return rc;
  }
  if (prec == 1 && !e->tc[0][0]) {
    if (Sh.empty()) {
      Sh.resize((size_t)e->n * e->n);
      CK(cudaMemcpy(Sh.data(), e->S, sizeof(double) * Sh.size(), cudaMemcpyDeviceToHost));
    }
    const int n = e->n, pitch = tc_pitch(n);
    for (int t = 0; t < 2; t++) {
      std::vector<float> hi((size_t)n * pitch, 0.0f), lo((size_t)n * pitch, 0.0f);
      for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++) {
          const double v = t == 0 ? Sh[(size_t)i * n + j] : Sh[(size_t)j * n + i];
          const float h = tf32_rna((float)v);
          hi[(size_t)i * pitch + j] = h;
          lo[(size_t)i * pitch + j] = (float)(v - (double)h);
        }
      for (int k = 0; k < 2; k++) {
        float* d = nullptr;
        if (int rc = dalloc(&d, hi.size())) return rc;
        CK(upload_now(d, k == 0 ? hi.data() : lo.data(), sizeof(float) * hi.size()));
        e->tc[t][k] = d;
      }
    }
    e->tc_pitch = pitch;
  }
  *out = e;
  return SE_OK;
}

// ---- Bloch form of a periodic direction (bloch.cu) ----
typedef std::complex<long double> cld;

// Eigenvalues and eigenvectors of a Hermitian n x n matrix (row-major, long
// double) by cyclic complex Jacobi rotations: each pivot's phase is moved
// into column q, then a real rotation (Numerical Recipes' tan formula)
// zeroes it. A is overwritten; U's columns are the eigenvectors. Jacobi in
// extended precision gives eigenvectors accurate to the FP64 rounding even
// for the small eigenvalues of these blocks, whose spread is about 1e5.
void herm_jacobi(int n, std::vector<cld>& A, std::vector<cld>& U, std::vector<long double>& ev) {
  U.assign((size_t)n * n, cld(0));
  for (int i = 0; i < n; i++) U[(size_t)i * n + i] = 1;
  for (int sweep = 0; sweep < 100; sweep++) {
    long double off = 0, dg = 0;
    for (int i = 0; i < n; i++)
      for (int j = 0; j < n; j++)
        (i == j ? dg : off) += std::norm(A[(size_t)i * n + j]);
    if (off <= 1e-36L * dg) break;
    for (int p = 0; p < n - 1; p++)
      for (int q = p + 1; q < n; q++) {
        const cld apq = A[(size_t)p * n + q];
        const long double r = std::abs(apq);
        if (r == 0) continue;
        const cld ph = apq / r, phc = std::conj(ph);
        for (int k = 0; k < n; k++) {
          A[(size_t)k * n + q] *= phc;  // column q by e^{-i phi}
          U[(size_t)k * n + q] *= phc;
        }
        for (int k = 0; k < n; k++) A[(size_t)q * n + k] *= ph;  // row q by e^{i phi}
        const long double app = A[(size_t)p * n + p].real(), aqq = A[(size_t)q * n + q].real();
        const long double th = (aqq - app) / (2 * r);
        const long double t = (th >= 0 ? 1 : -1) / (std::fabs(th) + std::sqrt(th * th + 1));
        const long double c = 1 / std::sqrt(t * t + 1), sn = t * c;
        for (int k = 0; k < n; k++) {
          const cld akp = A[(size_t)k * n + p], akq = A[(size_t)k * n + q];
          A[(size_t)k * n + p] = c * akp - sn * akq;
          A[(size_t)k * n + q] = sn * akp + c * akq;
          const cld ukp = U[(size_t)k * n + p], ukq = U[(size_t)k * n + q];
          U[(size_t)k * n + p] = c * ukp - sn * ukq;
          U[(size_t)k * n + q] = sn * ukp + c * ukq;
        }
        for (int k = 0; k < n; k++) {
          const cld apk = A[(size_t)p * n + k], aqk = A[(size_t)q * n + k];
          A[(size_t)p * n + k] = c * apk - sn * aqk;
          A[(size_t)q * n + k] = sn * apk + c * aqk;
        }
      }
  }
  ev.resize(n);
  for (int i = 0; i < n; i++) ev[i] = A[(size_t)i * n + i].real();
}

struct Bloch1D {
  BlochDir d;
  double2 *V = nullptr, *tw = nullptr;
  double* mu = nullptr;
};
std::mutex g_bloch_mu;
std::map<std::pair<int, int>, Bloch1D*> g_bloch[64];

// A periodic direction of 2^k >= 2 elements qualifies for the Bloch form
// when its transforms fit the kernels' 48 KB of shared memory (the y pass
// holds two complex copies of a column and the twiddles).
bool bloch_ok(const Dir& d) {
  return d.periodic && d.lo == 0 && d.nE >= 2 && (d.nE & (d.nE - 1)) == 0 &&
         16L * (2L * d.N * d.nE + d.nE / 2 + 1) <= 48L * 1024;
}

// The nel wavenumber blocks of one periodic direction (cached per device,
// element count and order): K_m and W_m from the reference element's
// stiffness Kh and weights w (the operator's coefficients scale them),
// W_m^{-1/2} K_m W_m^{-1/2} = U diag(mu) U^H by herm_jacobi, V = W^{-1/2} U.
int bloch_get(const Dir& d, const double* Kh, const double* w, Bloch1D** out) {
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return fail(SE_ERR_UNSUPPORTED, "device index %d", dev);
  std::lock_guard<std::mutex> lk(g_bloch_mu);
  Bloch1D*& b = g_bloch[dev][std::make_pair(d.nE, d.N)];
  if (b) {
    *out = b;
    return SE_OK;
  }
  const int nel = d.nE, p = d.N, n1 = p + 1;
  int logn = 0;
  while ((1 << logn) < nel) logn++;
  const long double two_pi = 6.283185307179586476925286766559005768L;
  std::vector<double2> V((size_t)nel * p * p), tw(std::max(1, nel / 2));
  std::vector<double> mu((size_t)nel * p);
  std::vector<long double> ws(p);
  for (int i = 0; i < p; i++) ws[i] = 1 / std::sqrt((long double)w[i] + (i == 0 ? w[p] : 0.0));
  std::vector<cld> A((size_t)p * p), U;
  std::vector<long double> ev;
  for (int m = 0; m < nel; m++) {
    const long double th = two_pi * m / nel;
    const cld eth(std::cos(th), std::sin(th));
    for (int i = 0; i < p; i++)
      for (int j = 0; j < p; j++) {
        cld v = (long double)Kh[i * n1 + j];
        if (i == 0 && j == 0) v += (long double)Kh[p * n1 + p];
        if (j == 0) v += (long double)Kh[i * n1 + p] * eth;
        if (i == 0) v += (long double)Kh[p * n1 + j] * std::conj(eth);
        A[(size_t)i * p + j] = ws[i] * v * ws[j];
      }
    herm_jacobi(p, A, U, ev);
    for (int i = 0; i < p; i++)
      for (int k = 0; k < p; k++) {
        const cld v = ws[i] * U[(size_t)i * p + k];
        V[((size_t)m * p + i) * p + k] = make_double2((double)v.real(), (double)v.imag());
      }
    for (int k = 0; k < p; k++) mu[(size_t)m * p + k] = (double)ev[k];
  }
  for (int j = 0; j < nel / 2; j++) {
    const long double a = two_pi * j / nel;
    tw[j] = make_double2((double)std::cos(a), (double)-std::sin(a));
  }
  Bloch1D* nb = new Bloch1D();
  int rc;
  if ((rc = dalloc(&nb->V, V.size())) || (rc = dalloc(&nb->tw, tw.size())) ||
      (rc = dalloc(&nb->mu, mu.size()))) {
    dfree(nb->V);
    dfree(nb->tw);
    dfree(nb->mu);
    delete nb;
    return rc;
  }
  CK(upload_now(nb->V, V.data(), sizeof(double2) * V.size()));
  CK(upload_now(nb->tw, tw.data(), sizeof(double2) * tw.size()));
  CK(upload_now(nb->mu, mu.data(), sizeof(double) * mu.size()));
  nb->d = BlochDir{nel, p, logn, nb->V, nb->mu, nb->tw};
  b = nb;
  *out = b;
  return SE_OK;
}

int fdm_setup(se_linsys* ls, int prec) {
  if (ls->svv)
    return fail(SE_ERR_UNSUPPORTED, "the SVV operator needs SE_METHOD_CG (no fast diagonalization)");
  if (ls->fdm_ready && ls->fdm_prec == prec) return SE_OK;
  const OpDev& op = ls->op;
  const size_t n = (size_t)ls->n;
  int rc;
  Eig1D *ex = nullptr, *ey = nullptr;
  if ((rc = eig_get(op.d[0], op.Kh, op.w, prec, &ex)) || (rc = eig_get(op.d[1], op.Kh, op.w, prec, &ey)))
    return rc;
  ls->Sx = ex->S;
  ls->Sy = ey->S;
  ls->SxT = ex->ST;
  ls->SyT = ey->ST;
  ls->lx = ex->lam;
  ls->ly = ey->lam;
  ls->lmax[0] = ex->lmax;
  ls->lmax[1] = ey->lmax;
  ls->Sx_lo = prec ? ex->low[prec] : nullptr;
  ls->Sy_lo = prec ? ey->low[prec] : nullptr;
  ls->SxT_lo = prec ? ex->lowT[prec] : nullptr;
  ls->SyT_lo = prec ? ey->lowT[prec] : nullptr;
  if (!ls->X1) {
    ls->fpart_n = std::max(kFdmPartials, std::max(residual_blocks(op), residual_partial_blocks(op)));
    if ((rc = dalloc(&ls->X1, n)) || (rc = dalloc(&ls->X2, n)) || (rc = dalloc(&ls->ax, n)) ||
        (rc = dalloc(&ls->zlow, 64)) || (rc = dalloc(&ls->fpart, 2 * (size_t)ls->fpart_n + 16)))
      return rc;
    ls->lowk = std::min(8, std::min(op.G[0], op.G[1]));
    if (bloch_ok(op.d[0]) && bloch_ok(op.d[1])) {
      Bloch1D *bx = nullptr, *by = nullptr;
      if ((rc = bloch_get(op.d[0], op.Kh, op.w, &bx)) || (rc = bloch_get(op.d[1], op.Kh, op.w, &by)))
        return rc;
      ls->bdx = bx->d;
      ls->bdy = by->d;
      if ((rc = dalloc(&ls->xh, bloch_spectrum_elems(ls->bdx, ls->bdy)))) return rc;
      ls->bloch = true;
    }
    // Jacobi inverse for the preconditioned residual norm
    CK(launch_op_diag(op, ls->dinv, g_stream));
    CK(launch_invert(ls->dinv, n, g_stream));
  }
  if (prec == 1) {
    for (int k = 0; k < 2; k++) {
      ls->tcSx[k] = ex->tc[0][k];
      ls->tcSxT[k] = ex->tc[1][k];
      ls->tcSy[k] = ey->tc[0][k];
      ls->tcSyT[k] = ey->tc[1][k];
    }
    ls->tc_px = ex->tc_pitch;
    ls->tc_py = ey->tc_pitch;
    if (!ls->tcY[0]) {
      const size_t ny = (size_t)op.G[1] * ls->tc_px, nx = (size_t)op.G[0] * ls->tc_py;
      for (int k = 0; k < 2; k++) {
        if ((rc = dalloc(&ls->tcY[k], ny)) || (rc = dalloc(&ls->tcX[k], nx))) return rc;
        CK(cudaMemsetAsync(ls->tcY[k], 0, sizeof(float) * ny, g_stream));
        CK(cudaMemsetAsync(ls->tcX[k], 0, sizeof(float) * nx, g_stream));
      }
      int dev = 0;
      CK(cudaGetDevice(&dev));
      CK(cudaDeviceGetAttribute(&ls->tc_sms, cudaDevAttrMultiProcessorCount, dev));
    }
  }
  if (prec == 2 && ls->fdm_lbuf_prec != prec) {
    const size_t es = prec == 1 ? sizeof(float) : sizeof(uint16_t);
    if (ls->L1) cudaFree(ls->L1);
    if (ls->L2) cudaFree(ls->L2);
    if (ls->L3) cudaFree(ls->L3);
    ls->L1 = ls->L2 = ls->L3 = nullptr;
    char *l2 = nullptr, *l3 = nullptr;
    if ((rc = dalloc(&l2, n * es)) || (rc = dalloc(&l3, n * es))) return rc;
    ls->L2 = l2;
    ls->L3 = l3;
    ls->fdm_lbuf_prec = prec;
  }
  ls->fdm_prec = prec;
  ls->fdm_ready = true;
  return SE_OK;
}

int op_gx(const se_linsys* ls) { return ls->op.G[0]; }
int op_gy(const se_linsys* ls) { return ls->op.G[1]; }

// Spectral entries below this magnitude are a null mode (constant null space
// of a periodic Poisson operator) and are zeroed.
double null_tol(const se_linsys* ls) {
  const OpDev& op = ls->op;
  return 1e-12 * (std::fabs(op.alpha) + std::fabs(op.beta[0]) * ls->lmax[0] +
                  std::fabs(op.beta[1]) * ls->lmax[1]);
}
// out (= or +=) A^{-1} in by four FP64 products on the row-major
// G_y x G_x unknown arrays F:  Ey^T (F Ex), spectral divide, then
// Ey ((.) Ex^T), the divide fused into the second product's epilogue and the
// accumulation into the fourth's (gemm.cu). The lowest lowk x lowk spectral
// block skips the backward products: the divide moves it to zlow and the
// fourth product adds Ey[:, <k] (zlow Ex[:, <k]^T) in double-double. For a
// smooth solution that block holds the largest coefficients, so the FP64
// rounding of the backward products no longer sets the first step's
// residual (with refined eigenvectors one step reaches about 3e-11 of the
// right-hand side in the Jacobi-preconditioned norm at 64x64 elements,
// p = 8, where plain FP64 products leave about 1e-9).
int fdm_apply64(se_linsys* ls, const double* in, double* out, bool accumulate,
                const FdmState* gate = nullptr) {
  const int gx = ls->op.G[0], gy = ls->op.G[1];
  const OpDev& op = ls->op;
  const double nt = null_tol(ls);
  if (ls->bloch) {
    CK(launch_bloch_inverse(ls->bdx, ls->bdy, op.alpha, op.beta[0], op.beta[1], nt, in, out,
                            accumulate, ls->xh, gate, g_stream));
    return SE_OK;
  }
  const FdmLow low{ls->zlow, ls->SxT, gx, ls->lowk};
  CK(launch_fdm_gemm(0, 0, in, 1, ls->SxT, ls->X1, 1, gy, gx, gx, gx, gx, gx, nullptr, nullptr,
                     nullptr, nullptr, 0, 0, 0, 0, g_stream, nullptr,
                     gate ? &gate->reason : nullptr));
  CK(launch_fdm_gemm(0, 1, ls->Sy, 1, ls->X1, ls->X2, 1, gy, gx, gy, gy, gx, gx, nullptr, nullptr,
                     ls->lx, ls->ly, op.alpha, op.beta[0], op.beta[1], nt, g_stream, &low));
  CK(launch_fdm_gemm(0, 0, ls->X2, 1, ls->Sx, ls->X1, 1, gy, gx, gx, gx, gx, gx, nullptr, nullptr,
                     nullptr, nullptr, 0, 0, 0, 0, g_stream));
  CK(launch_fdm_gemm(0, accumulate ? 2 : 0, ls->SyT, 1, ls->X1, out, 1, gy, gx, gy, gy, gx, gx,
                     nullptr, nullptr, nullptr, nullptr, 0, 0, 0, 0, g_stream, &low));
  return SE_OK;
}

// Low-precision x += A^{-1} in: the first product reads in scaled by
// 1/max|in| (max kept in device memory) and rounds it to the low type, the
// last adds its result back scaled by max. prec 1: FP32 data, TF32 tensor
// cores; prec 2: BF16 data; both accumulate in FP32.
int fdm_apply_low(se_linsys* ls, const double* in, double* out) {
  const int gx = ls->op.G[0], gy = ls->op.G[1];
  const size_t n = (size_t)gx * gy;
  const int prec = ls->fdm_prec;
  const OpDev& op = ls->op;
  double* mx = ls->fpart + 2 * ls->fpart_n;
  CK(launch_maxabs(in, n, ls->fpart, kFdmPartials, mx, g_stream));
  CK(launch_fdm_gemm(prec, 0, in, 1, ls->SxT_lo, ls->L2, 0, gy, gx, gx, gx, gx, gx, mx, nullptr,
                     nullptr, nullptr, 0, 0, 0, 0, g_stream));
  CK(launch_fdm_gemm(prec, 1, ls->Sy_lo, 0, ls->L2, ls->L3, 0, gy, gx, gy, gy, gx, gx, nullptr,
                     nullptr, ls->lx, ls->ly, op.alpha, op.beta[0], op.beta[1], null_tol(ls), g_stream));
  CK(launch_fdm_gemm(prec, 0, ls->L3, 0, ls->Sx_lo, ls->L2, 0, gy, gx, gx, gx, gx, gx, nullptr,
                     nullptr, nullptr, nullptr, 0, 0, 0, 0, g_stream));
  CK(launch_fdm_gemm(prec, 2, ls->SyT_lo, 0, ls->L2, out, 1, gy, gx, gy, gy, gx, gx, nullptr, mx,
                     nullptr, nullptr, 0, 0, 0, 0, g_stream));
  return SE_OK;
}


// x += A^{-1} r on the tcgen05 tensor cores (tc_gemm.cu): r split into TF32
// hi/lo pairs, then four products whose outputs chain without transposes
//   T1[x'][y] = F Ex,  T2[y'][x'] = (Ey^T T1) / lambda,  T3[x][y'] = T2 Ex^T,
//   x[y][x] += Ey T3,
// each product three TF32 MMAs per K step (about 21 operand bits), FP32
// accumulation; the last adds into the FP64 solution.
int fdm_apply_tc(se_linsys* ls, const double* in, double* out, bool split_done = false) {
  const int gx = ls->op.G[0], gy = ls->op.G[1];
  if (!ls->tc_plan || ls->tc_out != out) {
    // plans (tile shapes, tensor maps) of the four products, once per output
    const int px = ls->tc_px, py = ls->tc_py;
    const OpDev& op = ls->op;
    if (!ls->tc_plan) ls->tc_plan = new TcPlan[4];
    TcEpi e;
    std::memset(&e, 0, sizeof(e));
    e.err = &ls->d_fstate->kerr;
    // P1: M = gy, N = gx, K = gx
    e.M = gy; e.N = gx; e.K = gx; e.out_hi = ls->tcX[0]; e.out_lo = ls->tcX[1]; e.pitch = py;
    CK(tc_plan(&ls->tc_plan[0], TC_EPI_SPLIT, ls->tcY[0], ls->tcY[1], px, ls->tcSx[0], ls->tcSx[1],
               px, e));
    // P2: M = gx, N = gy, K = gy, spectral divide
    e.M = gx; e.N = gy; e.K = gy; e.out_hi = ls->tcY[0]; e.out_lo = ls->tcY[1]; e.pitch = px;
    e.lm = ls->lx; e.ln = ls->ly; e.alpha = op.alpha; e.bm = op.beta[0]; e.bn = op.beta[1];
    e.null_tol = null_tol(ls);
    CK(tc_plan(&ls->tc_plan[1], TC_EPI_DIVIDE, ls->tcX[0], ls->tcX[1], py, ls->tcSy[0],
               ls->tcSy[1], py, e));
    // P3: M = gy, N = gx, K = gx
    e.M = gy; e.N = gx; e.K = gx; e.out_hi = ls->tcX[0]; e.out_lo = ls->tcX[1]; e.pitch = py;
    CK(tc_plan(&ls->tc_plan[2], TC_EPI_SPLIT, ls->tcY[0], ls->tcY[1], px, ls->tcSxT[0],
               ls->tcSxT[1], px, e));
    // P4: M = gx, N = gy, K = gy, accumulated into the FP64 solution [gy][gx]
    e.M = gx; e.N = gy; e.K = gy; e.out_hi = e.out_lo = nullptr; e.out64 = out; e.pitch = gx;
    CK(tc_plan(&ls->tc_plan[3], TC_EPI_ACC64, ls->tcX[0], ls->tcX[1], py, ls->tcSyT[0],
               ls->tcSyT[1], py, e));
    ls->tc_out = out;
  }
  // the input's TF32 split (the refinement loop's residual kernel writes it)
  if (!split_done) CK(launch_tc_split(in, gy, gx, gx, ls->tcY[0], ls->tcY[1], ls->tc_px, g_stream));
  for (int k = 0; k < 4; k++) CK(launch_tc_plan(ls->tc_plan[k], g_stream));
  return SE_OK;
}

// The whole FDM solve as one CUDA graph: right-hand side assembly, r = f,
// x = 0, the initial norm and test, then a conditional while-node whose body
// refines x += A^{-1} r, forms r = f - A x with its norm and runs the
// convergence test that sets the loop condition; finally the field update.
// Parameters (rtol, atol, dtol, max_it) and the loop state live in device
// memory, so one solve is one graph launch and one read of the state.
// Node and edge kinds of a captured graph, for error messages.
std::string describe_graph(cudaGraph_t g) {
  if (!g) return "none";
  size_t nn = 0;
  if (cudaGraphGetNodes(g, nullptr, &nn) != cudaSuccess) return "?";
  std::vector<cudaGraphNode_t> nodes(nn);
  cudaGraphGetNodes(g, nodes.data(), &nn);
  int kinds[16] = {0}, clusters = 0, pdl_attr = 0;
  for (auto nd : nodes) {
    cudaGraphNodeType t;
    if (cudaGraphNodeGetType(nd, &t) != cudaSuccess) continue;
    kinds[(int)t & 15]++;
    if (t == cudaGraphNodeTypeKernel) {
      cudaLaunchAttributeValue v;
      if (cudaGraphKernelNodeGetAttribute(nd, cudaLaunchAttributeClusterDimension, &v) == cudaSuccess &&
          v.clusterDim.x * v.clusterDim.y * v.clusterDim.z > 1)
        clusters++;
      if (cudaGraphKernelNodeGetAttribute(nd, cudaLaunchAttributeProgrammaticStreamSerialization, &v) == cudaSuccess &&
          v.programmaticStreamSerializationAllowed)
        pdl_attr++;
    }
  }
  size_t ne = 0;
  int prog = 0;
  if (cudaGraphGetEdges_v2(g, nullptr, nullptr, nullptr, &ne) == cudaSuccess && ne) {
    std::vector<cudaGraphNode_t> from(ne), to(ne);
    std::vector<cudaGraphEdgeData> ed(ne);
    if (cudaGraphGetEdges_v2(g, from.data(), to.data(), ed.data(), &ne) == cudaSuccess)
      for (size_t k = 0; k < ne; k++)
        if (ed[k].type != cudaGraphDependencyTypeDefault) prog++;
  }
  cudaGetLastError();
  char buf[256];
  snprintf(buf, sizeof(buf),
           "%zu nodes: %d kernel, %d memcpy, %d memset, %d host, %d graph, %d empty, %d other; "
           "%d clustered, %d with programmatic serialization; %zu edges, %d programmatic",
           nn, kinds[cudaGraphNodeTypeKernel], kinds[cudaGraphNodeTypeMemcpy],
           kinds[cudaGraphNodeTypeMemset], kinds[cudaGraphNodeTypeHost], kinds[cudaGraphNodeTypeGraph],
           kinds[cudaGraphNodeTypeEmpty],
           (int)nn - kinds[cudaGraphNodeTypeKernel] - kinds[cudaGraphNodeTypeMemcpy] -
               kinds[cudaGraphNodeTypeMemset] - kinds[cudaGraphNodeTypeHost] -
               kinds[cudaGraphNodeTypeGraph] - kinds[cudaGraphNodeTypeEmpty],
           clusters, pdl_attr, ne, prog);
  return buf;
}

int fdm_build_graph(se_linsys* ls, int prec, int remove_null) {
  if (!ls->d_fparams) {
    int rc;
    if ((rc = dalloc(&ls->d_fparams, 1)) || (rc = dalloc(&ls->d_fstate, 1)) ||
        (rc = dalloc(&ls->d_rescount, 1)))
      return rc;
    CK(cudaMemsetAsync(ls->d_rescount, 0, sizeof(unsigned), g_stream));
  }
  if (ls->fdm_exec) {
    cudaGraphExecDestroy(ls->fdm_exec);
    ls->fdm_exec = nullptr;
  }
  const cudaStream_t saved = g_stream;
  cudaStream_t cs = nullptr, bs = nullptr;
  CK(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
  CK(cudaStreamCreateWithFlags(&bs, cudaStreamNonBlocking));
  auto cleanup = [&]() {
    g_stream = saved;
    cudaStreamDestroy(cs);
    cudaStreamDestroy(bs);
  };
  int rc = SE_OK;
  cudaGraph_t graph = nullptr;
  do {
    const MeshDev& m = ls->sol->mesh->dev;
    const size_t n = (size_t)ls->n;
    const int nt = ls->opts.norm_type;
    const double* wv = nt == SE_NORM_UNPRECONDITIONED ? nullptr : ls->dinv;
    double* res = ls->fpart + 2 * ls->fpart_n + 2;
    g_stream = cs;
    cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) { rc = cuda_fail(e, "begin capture"); break; }
    cudaStreamCaptureStatus status;
    cudaGraph_t cg = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    // the while loop's condition hc: set by the initial test and by each
    // step's test (prec 3: FP64 first step, tensor-core steps after)
    cudaGraphConditionalHandle hc;
    bool ok = cudaStreamGetCaptureInfo(cs, &status, nullptr, &cg, &deps, &ndeps) == cudaSuccess &&
              cudaGraphConditionalHandleCreate(&hc, cg, 0, 0) == cudaSuccess;
    // prologue: without a null space to remove and with an FP64 first
    // inverse, one launch (f, r = f, x = 0, the initial norm and test);
    // otherwise the pieces one by one
    if (!remove_null && prec != 1) {
      ok = ok && launch_fdm_prologue(ls->op, m, ls->rhs ? ls->rhs->vals : nullptr, ls->lift, ls->f,
                                     ls->r, ls->x, wv, nt == SE_NORM_NATURAL, ls->fpart,
                                     kFdmPartials, res, ls->d_rescount, ls->d_fparams,
                                     ls->d_fstate, hc, cs) == cudaSuccess;
    } else {
      ok = ok && launch_rhs_assemble(ls->op, m, ls->rhs ? ls->rhs->vals : nullptr, ls->lift, ls->f, cs) == cudaSuccess;
      // a right-hand side off the range of a singular operator: solve for the
      // one Jacobi CG with the null space removed converges to
      if (remove_null)
        ok = ok && launch_project_null(ls->f, ls->dinv, n, ls->fpart, kFdmPartials,
                                       ls->fpart + 2 * ls->fpart_n + 4, cs) == cudaSuccess;
      ok = ok && cudaMemcpyAsync(ls->r, ls->f, sizeof(double) * n, cudaMemcpyDeviceToDevice, cs) == cudaSuccess;
      // the tensor-core inverse reads r as TF32 hi/lo pairs: the first from f,
      // the others from the residual kernel
      if (prec == 1)
        ok = ok && launch_tc_split(ls->f, op_gy(ls), op_gx(ls), op_gx(ls), ls->tcY[0], ls->tcY[1],
                                   ls->tc_px, cs) == cudaSuccess;
      ok = ok && cudaMemsetAsync(ls->x, 0, sizeof(double) * n, cs) == cudaSuccess;
      ok = ok && launch_norms(ls->f, wv, n, nt == SE_NORM_NATURAL, ls->fpart, kFdmPartials, res, cs) == cudaSuccess;
      ok = ok && launch_fdm_init(ls->d_fparams, ls->d_fstate, res, hc, cs) == cudaSuccess;
    }
    // a conditional node after what was captured so far, its body captured on
    // stream bs by `fill`
    std::vector<cudaGraph_t> bodies;
    auto add_cond = [&](cudaGraphConditionalHandle h, cudaGraphConditionalNodeType type,
                        const std::function<int()>& fill) {
      if (!ok) return;
      cudaGraphNode_t cn = nullptr;
      ok = cudaStreamGetCaptureInfo(cs, &status, nullptr, &cg, &deps, &ndeps) == cudaSuccess;
      cudaGraphNodeParams cp = {};
      cp.type = cudaGraphNodeTypeConditional;
      cp.conditional.handle = h;
      cp.conditional.type = type;
      cp.conditional.size = 1;
      ok = ok && cudaGraphAddNode(&cn, cg, deps, ndeps, &cp) == cudaSuccess;
      ok = ok && cudaStreamUpdateCaptureDependencies(cs, &cn, 1, cudaStreamSetCaptureDependencies) == cudaSuccess;
      if (!ok) return;
      cudaGraph_t body = cp.conditional.phGraph_out[0];
      bodies.push_back(body);
      g_stream = bs;
      ok = cudaStreamBeginCaptureToGraph(bs, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
      if (ok) {
        const int brc = fill();
        cudaGraph_t bodyg = body;
        const bool ended = cudaStreamEndCapture(bs, &bodyg) == cudaSuccess;
        ok = ended && brc == SE_OK;
      }
      g_stream = cs;
    };
    // one refinement step: x += A^{-1} r with the given inverse, then r = f - A x
    // with the norm and the convergence test (setting hc) in one launch, and
    // the TF32 split of r when tensor-core steps follow
    // (gate: the loop state that makes an unconditional first step add
    // nothing when the initial test has already decided)
    auto step = [&](int inv, const FdmState* gate) -> int {
      int brc = inv == 0   ? fdm_apply64(ls, ls->r, ls->x, true, gate)
                : inv == 1 ? fdm_apply_tc(ls, ls->r, ls->x, true)
                           : fdm_apply_low(ls, ls->r, ls->x);
      if (!brc && remove_null)
        brc = launch_remove_mean(ls->x, n, ls->fpart, kFdmPartials, ls->fpart + 2 * ls->fpart_n + 4, bs) == cudaSuccess ? SE_OK : SE_ERR_CUDA;
      const bool split = prec == 1 || prec == 3;
      if (!brc)
        brc = launch_residual_check(ls->op, ls->x, ls->f, ls->r, wv, nt == SE_NORM_NATURAL,
                                    ls->fpart, res, ls->d_rescount, ls->d_fparams, ls->d_fstate,
                                    hc, bs, split ? ls->tcY[0] : nullptr,
                                    split ? ls->tcY[1] : nullptr, ls->tc_px) == cudaSuccess
                  ? SE_OK
                  : SE_ERR_CUDA;
      return brc;
    };
    // An FP64 first step (prec 0 and 3) as plain nodes of the graph (most
    // solves need only it), the loop for the rest: the conditional node
    // cost about 4 us a solve at 64x64 elements, p = 8. A step whose
    // initial test has decided adds nothing: its first pass (the Bloch x
    // pass, or the first dense product) takes the residual as zero, and its
    // test keeps the decision and the count.
    if ((prec == 0 || prec == 3) && ok) {
      const cudaStream_t body_stream = bs;
      bs = cs;
      ok = step(0, ls->d_fstate) == SE_OK;
      bs = body_stream;
    }
    add_cond(hc, cudaGraphCondTypeWhile, [&]() { return step(prec == 3 ? 1 : prec, nullptr); });
    cudaGraph_t body = bodies.empty() ? nullptr : bodies.back();
    // epilogue
    // (and the loop state to the mapped host buffer, when there is one)
    ok = ok && launch_update_field(ls->op, m, ls->x, ls->sol->vals, cs, ls->d_fstate,
                                   ls->h_fstate_dev) == cudaSuccess;
    const bool ended = cudaStreamEndCapture(cs, &graph) == cudaSuccess;
    if (!ok || !ended) {
      cudaGetLastError();
      rc = fail(SE_ERR_CUDA, "capturing the FDM solve graph failed");
      break;
    }
    e = cudaGraphInstantiate(&ls->fdm_exec, graph, 0);
    if (e != cudaSuccess) {
      rc = fail(SE_ERR_CUDA, "cudaGraphInstantiate: %s (loop body: %s)", cudaGetErrorString(e),
                describe_graph(body).c_str());
      cudaGetLastError();
      ls->fdm_exec = nullptr;
      break;
    }
    ls->fdm_key = prec | (remove_null << 2) | (nt << 3) | (ls->opts.mode << 6);
    ls->fdm_state_mapped = ls->h_fstate_dev != nullptr;
  } while (0);
  if (graph) cudaGraphDestroy(graph);
  cleanup();
  return rc;
}

// Queue the FDM solve of A x = f (fast diagonalization with FP64 iterative
// refinement until the chosen residual norm is <= max(rtol |f|, atol)) on the
// calling thread's stream: parameter upload, the solve graph (right-hand side
// assembly through the field update) and the state read-back into pinned
// memory. fdm_finish reads the state once the stream is done.
// The loop's parameters go up when they differ from the last upload, or
// always with upload_params (the batch path: on a B200 its 256-solve
// ensemble, graphs round-robin on 8 streams, ran 5.1 ms with the upload
// before every graph and 7.5 ms without it; a single solve is 3 us faster
// without it).
int fdm_launch(se_linsys* ls, int remove_null, bool upload_params) {
  // inverse kinds: 0 FP64, 1 TF32x3 tensor cores, 2 BF16, 3 FP64 first then 1
  const int pr = ls->opts.precision;
  const int prec = pr == SE_PREC_FP64 ? 0 : pr == SE_PREC_MIXED ? 1 : pr == SE_PREC_FP64_TC ? 3 : 2;
  if (int rc = fdm_setup(ls, prec == 3 ? 1 : prec)) return rc;
  const int key = prec | ((remove_null != 0) << 2) | (ls->opts.norm_type << 3) | (ls->opts.mode << 6);
  if (!ls->h_fparams) {
    // page-locked and mapped: the state comes back through the graph's last
    // kernel instead of a copy; a buffer that cannot be mapped falls back to
    // the copy
    void* p = nullptr;
    CK(cudaHostAlloc(&p, sizeof(FdmParams) + sizeof(FdmState), cudaHostAllocMapped));
    ls->h_fparams = static_cast<FdmParams*>(p);
    ls->h_fstate = reinterpret_cast<FdmState*>(ls->h_fparams + 1);
    void* dp = nullptr;
    if (cudaHostGetDevicePointer(&dp, p, 0) == cudaSuccess && dp)
      ls->h_fstate_dev = reinterpret_cast<FdmState*>(static_cast<FdmParams*>(dp) + 1);
    else
      cudaGetLastError();
  }
  if (!ls->fdm_exec || ls->fdm_key != key)
    if (int rc = fdm_build_graph(ls, prec, remove_null != 0)) return rc;
  if (!ls->ev[2]) {
    for (cudaEvent_t& e : ls->ev)
      if (!e) CK(cudaEventCreate(&e));
  }
  FdmParams p;
  std::memset(&p, 0, sizeof(p));
  p.rtol = ls->opts.rtol;
  p.atol = ls->opts.atol;
  p.dtol = ls->opts.dtol;
  p.max_it = ls->opts.max_it;
  if (upload_params || !ls->fparams_sent || std::memcmp(&p, &ls->fparams_last, sizeof(p)) != 0) {
    *ls->h_fparams = p;
    CK(cudaMemcpyAsync(ls->d_fparams, ls->h_fparams, sizeof(FdmParams), cudaMemcpyHostToDevice, g_stream));
    ls->fparams_last = p;
    ls->fparams_sent = true;
  }
  CK(cudaEventRecord(ls->ev[0], g_stream));
  CK(cudaGraphLaunch(ls->fdm_exec, g_stream));
  CK(cudaEventRecord(ls->ev[1], g_stream));
  if (!ls->fdm_state_mapped)
    CK(cudaMemcpyAsync(ls->h_fstate, ls->d_fstate, sizeof(FdmState), cudaMemcpyDeviceToHost, g_stream));
  CK(cudaEventRecord(ls->ev[2], g_stream));
  return SE_OK;
}
int fdm_finish(se_linsys* ls, CgSolve* st, float* kernel_ms) {
  CK(cudaEventSynchronize(ls->ev[2]));  // the state has reached the host
  if (kernel_ms) CK(cudaEventElapsedTime(kernel_ms, ls->ev[0], ls->ev[1]));
  std::memset(st, 0, sizeof(*st));
  st->its = ls->h_fstate->its;
  st->reason = ls->h_fstate->reason;
  st->dp = ls->h_fstate->dp;
  st->rnorm0 = ls->h_fstate->rnorm0;
  if (ls->h_fstate->kerr & KERR_BARRIER_TIMEOUT)
    return fail(SE_ERR_TIMEOUT, "FDM solve: a tensor-core product's bounded wait gave up");
  return SE_OK;
}
int run_fdm(se_linsys* ls, int remove_null, CgSolve* st, float* kernel_ms) {
  if (int rc = fdm_launch(ls, remove_null, false)) return rc;
  CK(cudaStreamSynchronize(g_stream));
  return fdm_finish(ls, st, kernel_ms);
}

// ---------------------------------------------------------- batched CG ----
// Workspace of batched CG launches (grow-only, per device).
struct BatchWs {
  CgSolve* solves = nullptr;
  CgTile* tiles = nullptr;
  int* begin = nullptr;
  double* partials = nullptr;
  unsigned* words = nullptr;  // barrier, error
  size_t cap_solves = 0, cap_tiles = 0, cap_begin = 0, cap_part = 0;
  std::vector<CgSolve> h_solves;
};
std::mutex g_batch_mu;
BatchWs g_batch[64];

template <class T>
int grow(T** p, size_t* cap, size_t need) {
  if (*cap >= need) return SE_OK;
  if (*p) cudaFree(*p);
  *p = nullptr;
  *cap = 0;
  size_t n = std::max(need, (size_t)(*cap * 2));
  if (int rc = dalloc(p, n)) return rc;
  *cap = n;
  return SE_OK;
}

// Launch-shape autotuner for batched CG: for a batch signature (order,
// number of solves, tile count rounded up to a power of two) it times short
// capped runs (30 iterations) of each candidate -- the register-resident
// mode when it fits, and the streaming mode at 1, 2 and 4 blocks per SM --
// and keeps the fastest. Decisions are cached for the process.
struct TuneChoice {
  bool resident;
  int grid;
};
std::mutex g_tune_mu;
std::map<std::tuple<int, int, int, int>, TuneChoice> g_tune;

int run_cg_batch_once(int dev, std::vector<se_linsys*>& sys, const std::vector<const OpDev*>& ops,
                      int N, bool resident, int grid, int max_it_cap, int remove_null, float* ms) {
  BatchWs& W = g_batch[dev];
  Schedule S = make_schedule(ops, grid);
  const int g = (int)S.block_begin.size() - 1;
  const size_t ns = sys.size();
  int rc;
  if ((rc = grow(&W.solves, &W.cap_solves, ns)) || (rc = grow(&W.tiles, &W.cap_tiles, S.tiles.size())) ||
      (rc = grow(&W.begin, &W.cap_begin, S.block_begin.size())) ||
      (rc = grow(&W.partials, &W.cap_part, (size_t)S.nseg * 8)))
    return rc;
  if (!W.words && (rc = dalloc(&W.words, 64))) return rc;
  W.h_solves.resize(ns);
  for (size_t i = 0; i < ns; i++) {
    se_linsys* ls = sys[i];
    CgSolve& cs = W.h_solves[i];
    cs = make_solve(ls, ls->f, ls->x, ls->opts.rtol, ls->opts.atol, ls->opts.dtol,
                    max_it_cap > 0 ? std::min(max_it_cap, ls->opts.max_it) : ls->opts.max_it, remove_null);
    cs.seg_begin = S.seg_begin[i];
    cs.seg_end = S.seg_end[i];
  }
  cudaStream_t s = g_stream;
  CK(cudaMemcpyAsync(W.solves, W.h_solves.data(), sizeof(CgSolve) * ns, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(W.tiles, S.tiles.data(), sizeof(CgTile) * S.tiles.size(), cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(W.begin, S.block_begin.data(), sizeof(int) * S.block_begin.size(), cudaMemcpyHostToDevice, s));
  CK(cudaMemsetAsync(W.words, 0, 64 * sizeof(unsigned), s));
  CgBatch B;
  B.solves = W.solves;
  B.nsolves = (int)ns;
  B.tiles = W.tiles;
  B.block_tile_begin = W.begin;
  B.partials = W.partials;
  B.nseg = S.nseg;
  B.bar_count = W.words;
  B.bar_gen = W.words + 32;
  B.n_active = reinterpret_cast<int*>(W.words + 40);
  B.err = W.words + 48;
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  CK(cudaEventRecord(e0, s));
  cudaError_t le = launch_cg(B, g, N, resident, s);
  CK(cudaEventRecord(e1, s));
  CK(cudaMemcpyAsync(W.h_solves.data(), W.solves, sizeof(CgSolve) * ns, cudaMemcpyDeviceToHost, s));
  unsigned err = 0;
  CK(cudaMemcpyAsync(&err, B.err, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  if (ms) cudaEventElapsedTime(ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (le != cudaSuccess) return cuda_fail(le, "batched CG launch");
  if (err & KERR_BARRIER_TIMEOUT) return fail(SE_ERR_TIMEOUT, "CG grid barrier timed out");
  return SE_OK;
}

int solve_cg_group(std::vector<se_linsys*>& sys, int remove_null, std::vector<CgSolve>& out, float* ms) {
  int dev = 0;
  CK(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(g_batch_mu);
  const int N = sys[0]->op.d[0].N;
  std::vector<const OpDev*> ops;
  long ntiles = 0;
  for (se_linsys* ls : sys) {
    ops.push_back(&ls->op);
    ntiles += cg_tiles(ls->op);
  }
  int bucket = 1;
  while (bucket < ntiles) bucket <<= 1;
  const auto key = std::make_tuple(dev, N, (int)sys.size(), bucket);
  TuneChoice choice{false, 0};
  bool have = false;
  {
    std::lock_guard<std::mutex> tl(g_tune_mu);
    auto it = g_tune.find(key);
    if (it != g_tune.end()) {
      choice = it->second;
      have = true;
    }
  }
  if (!have) {
    int sms = 1;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    std::vector<TuneChoice> cands;
    const int maxr = cg_max_grid(dev, N, true, (int)sys.size());
    if (maxr > 0 && ntiles <= (long)maxr * kCgResidentTiles)
      cands.push_back({true, (int)std::min<long>(maxr, ntiles)});
    const int maxs = cg_max_grid(dev, N, false, (int)sys.size());
    for (int per : {1, 2, 4})
      if (maxs > 0 && sms * per <= maxs) cands.push_back({false, (int)std::min<long>(sms * per, ntiles)});
    if (cands.empty()) return fail(SE_ERR_CUDA, "no co-resident launch shape for the batched CG");
    float best = 1e30f;
    for (const TuneChoice& c : cands) {
      float t = 0.f;
      if (int rc = run_cg_batch_once(dev, sys, ops, N, c.resident, c.grid, 30, remove_null, &t)) return rc;
      if (t < best) {
        best = t;
        choice = c;
      }
    }
    std::lock_guard<std::mutex> tl(g_tune_mu);
    g_tune[key] = choice;
  }
  if (int rc = run_cg_batch_once(dev, sys, ops, N, choice.resident, choice.grid, 0, remove_null, ms))
    return rc;
  out.assign(g_batch[dev].h_solves.begin(), g_batch[dev].h_solves.begin() + sys.size());
  return SE_OK;
}
}  // namespace

// =========================================================== C-ABI ========
extern "C" {

const char* se_last_error(void) { return g_err.c_str(); }
const char* se_version(void) { return "segpu 0.1 (sm_100a)"; }

int se_set_stream(void* stream) {
  g_stream = (cudaStream_t)stream;
  return SE_OK;
}
int se_synchronize(void) {
  CK(cudaStreamSynchronize(g_stream));
  return SE_OK;
}

// ---------------------------------------------------------------- mesh ----
int se_mesh_create(const int nEls[2], int N, const double min[2], const double max[2],
                   const int periodic[2], se_mesh** out) {
  if (!out || !nEls || !min || !max || !periodic) return fail(SE_ERR_ARG, "null argument");
  *out = nullptr;
  if (N < 2 || N > SE_MAXN)
    return fail(SE_ERR_UNSUPPORTED, "polynomial order %d outside [2, %d]", N, SE_MAXN);
  if (nEls[0] < 1 || nEls[1] < 1) return fail(SE_ERR_ARG, "element counts must be positive");
  if (!(max[0] > min[0]) || !(max[1] > min[1])) return fail(SE_ERR_ARG, "empty domain");
  long nv = (long)(nEls[0] * (long)N + 1) * (nEls[1] * (long)N + 1);
  if (nv > (1L << 30)) return fail(SE_ERR_UNSUPPORTED, "mesh too large");
  se_mesh* m = new se_mesh();
  gll_build(N, m->gll);
  MeshDev& d = m->dev;
  std::memset(&d, 0, sizeof(d));
  d.N = N;
  for (int k = 0; k < 2; k++) {
    d.nEls[k] = nEls[k];
    d.nVerts[k] = nEls[k] * N + 1;
    d.periodic[k] = periodic[k] != 0;
    d.min[k] = min[k];
    d.max[k] = max[k];
    d.dx[k] = (d.max[k] - d.min[k]) / d.nEls[k];
    d.two_over_dx[k] = 2.0 / d.dx[k];
    d.span[k] = d.max[k] - d.min[k];
    d.nspan[k] = d.min[k] - d.max[k];
  }
  for (int i = 0; i <= N; i++) {
    d.abcissa[i] = m->gll.x[i];
    d.lambda[i] = m->gll.lambda[i];
    d.w[i] = m->gll.w[i];
  }
  for (int i = 0; i < (N + 1) * (N + 1); i++) d.dC[i] = m->gll.dC[i];
  m->nVertsTotal = d.nVerts[0] * d.nVerts[1];
  *out = m;
  return SE_OK;
}
int se_mesh_destroy(se_mesh* mesh) {
  delete mesh;
  return SE_OK;
}
int se_mesh_sizes(const se_mesh* mesh, int nVerts[2], int* nVertsTotal) {
  if (!mesh) return fail(SE_ERR_ARG, "null mesh");
  if (nVerts) {
    nVerts[0] = mesh->dev.nVerts[0];
    nVerts[1] = mesh->dev.nVerts[1];
  }
  if (nVertsTotal) *nVertsTotal = mesh->nVertsTotal;
  return SE_OK;
}
int se_mesh_verts(const se_mesh* mesh, double* verts) {
  if (!mesh || !verts) return fail(SE_ERR_ARG, "null argument");
  const MeshDev& d = mesh->dev;
  for (int v = 0; v < mesh->nVertsTotal; v++) {
    int t[2] = {v % d.nVerts[0], v / d.nVerts[0]};
    for (int k = 0; k < 2; k++) {
      int e = t[k] / d.N;
      double l = d.abcissa[t[k] % d.N];
      verts[2 * v + k] = d.min[k] + e * d.dx[k] + ((l + 1.0) / 2.0) * d.dx[k];
    }
  }
  return SE_OK;
}
int se_mesh_gll(const se_mesh* mesh, double* abcissa, double* weights, double* dCij) {
  if (!mesh) return fail(SE_ERR_ARG, "null mesh");
  const int n = mesh->dev.N + 1;
  if (abcissa) std::memcpy(abcissa, mesh->gll.x, sizeof(double) * n);
  if (weights) std::memcpy(weights, mesh->gll.w, sizeof(double) * n);
  if (dCij) std::memcpy(dCij, mesh->gll.dC, sizeof(double) * n * n);
  return SE_OK;
}
int se_mesh_global_to_local(const se_mesh* mesh, const double* pts, int npts, int* el,
                            double* lcoord) {
  if (!mesh || npts < 0 || (npts && (!pts || !el || !lcoord)))
    return fail(SE_ERR_ARG, "bad argument");
  if (npts == 0) return SE_OK;
  double *dp = nullptr, *dl = nullptr;
  int* de = nullptr;
  int rc;
  if ((rc = dalloc(&dp, 2 * (size_t)npts)) || (rc = dalloc(&dl, 2 * (size_t)npts)) ||
      (rc = dalloc(&de, npts))) {
    dfree(dp);
    dfree(dl);
    dfree(de);
    return rc;
  }
  cudaStream_t s = g_stream;
  cudaError_t e = cudaMemcpyAsync(dp, pts, sizeof(double) * 2 * npts, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = launch_global_to_local(mesh->dev, dp, npts, de, dl, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(el, de, sizeof(int) * npts, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(lcoord, dl, sizeof(double) * 2 * npts, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  dfree(dp);
  dfree(dl);
  dfree(de);
  if (e != cudaSuccess) return cuda_fail(e, "global_to_local");
  return SE_OK;
}

// ----------------------------------------------------------------- bcs ----
int se_bcs_create(se_mesh* mesh, int bottom, int top, int left, int right, se_bcs** out) {
  if (!mesh || !out) return fail(SE_ERR_ARG, "null argument");
  *out = nullptr;
  const MeshDev& m = mesh->dev;
  bool b = bottom != 0, t = top != 0, l = left != 0, r = right != 0;
  // src/base/BCs.cpp:51-58: periodic and wall conditions exclude each other
  if ((b || t) && m.periodic[1])
    return fail(SE_ERR_ARG, "both periodic and non-periodic conditions in y");
  if ((l || r) && m.periodic[0])
    return fail(SE_ERR_ARG, "both periodic and non-periodic conditions in x");
  // src/base/BCs.cpp:113-194: the reference builds maps for no/full
  // periodicity and for periodicity in x only.
  if (m.periodic[1] && !m.periodic[0])
    return fail(SE_ERR_UNSUPPORTED, "periodic in y only is not built by the reference");
  if (m.periodic[0] && !m.periodic[1] && b && !t)
    return fail(SE_ERR_UNSUPPORTED, "periodic x with a bottom wall only (reference: bc error)");
  se_bcs* bc = new se_bcs();
  bc->mesh = mesh;
  bc->bottom = b;
  bc->top = t || m.periodic[1];
  bc->left = l;
  bc->right = r || m.periodic[0];
  bc->d[0] = make_dir(m, 0, l, r);
  bc->d[1] = make_dir(m, 1, b, t);
  bc->vec_size = (bc->d[0].hi - bc->d[0].lo) * (bc->d[1].hi - bc->d[1].lo);
  *out = bc;
  return SE_OK;
}
int se_bcs_destroy(se_bcs* bcs) {
  delete bcs;
  return SE_OK;
}
int se_bcs_vec_size(const se_bcs* bcs, int* n) {
  if (!bcs || !n) return fail(SE_ERR_ARG, "null argument");
  *n = bcs->vec_size;
  return SE_OK;
}
int se_bcs_maps(const se_bcs* bcs, int* field_to_vec, int* vec_to_field) {
  if (!bcs) return fail(SE_ERR_ARG, "null bcs");
  const MeshDev& m = bcs->mesh->dev;
  const Dir &dx = bcs->d[0], &dy = bcs->d[1];
  const int G0 = dx.hi - dx.lo, nvx = m.nVerts[0], nvy = m.nVerts[1];
  for (int j = 0; j < nvy; j++)
    for (int i = 0; i < nvx; i++) {
      int gi = (dx.periodic && i == nvx - 1) ? 0 : i;
      int gj = (dy.periodic && j == nvy - 1) ? 0 : j;
      bool in = gi >= dx.lo && gi < dx.hi && gj >= dy.lo && gj < dy.hi;
      int v = in ? (gj - dy.lo) * G0 + (gi - dx.lo) : -1;
      if (field_to_vec) field_to_vec[j * nvx + i] = v;
      if (vec_to_field && in && gi == i && gj == j) vec_to_field[v] = j * nvx + i;
    }
  return SE_OK;
}

// --------------------------------------------------------------- field ----
int se_field_create(se_mesh* mesh, int ndofs, se_bcs* bcs, se_field** out) {
  if (!mesh || !out) return fail(SE_ERR_ARG, "null argument");
  *out = nullptr;
  if (ndofs < 1 || ndofs > 2) return fail(SE_ERR_UNSUPPORTED, "ndofs %d not in [1, 2]", ndofs);
  if (bcs && bcs->mesh != mesh) return fail(SE_ERR_ARG, "bcs built on another mesh");
  if (int rc = ensure_globals()) return rc;
  se_field* f = new se_field();
  f->mesh = mesh;
  f->ndofs = ndofs;
  f->bcs = bcs;
  int rc = dalloc(&f->vals, (size_t)mesh->nVertsTotal * ndofs);
  if (rc) {
    delete f;
    return rc;
  }
  cudaError_t e = cudaMemsetAsync(f->vals, 0, sizeof(double) * mesh->nVertsTotal * ndofs, g_stream);
  if (e != cudaSuccess) {
    dfree(f->vals);
    delete f;
    return cuda_fail(e, "cudaMemset");
  }
  *out = f;
  return SE_OK;
}
int se_field_destroy(se_field* field) {
  if (!field) return SE_OK;
  dfree(field->vals);
  delete field;
  return SE_OK;
}
int se_field_upload(se_field* field, const double* vals) {
  if (int rc = check_field(field)) return rc;
  if (!vals) return fail(SE_ERR_ARG, "null host array");
  CK(cudaMemcpyAsync(field->vals, vals, sizeof(double) * field->mesh->nVertsTotal * field->ndofs,
                     cudaMemcpyHostToDevice, g_stream));
  return SE_OK;
}
int se_field_download(const se_field* field, double* vals) {
  if (int rc = check_field(field)) return rc;
  if (!vals) return fail(SE_ERR_ARG, "null host array");
  CK(cudaMemcpyAsync(vals, field->vals, sizeof(double) * field->mesh->nVertsTotal * field->ndofs,
                     cudaMemcpyDeviceToHost, g_stream));
  CK(cudaStreamSynchronize(g_stream));
  return SE_OK;
}
int se_field_download_async(const se_field* field, double* vals) {
  if (int rc = check_field(field)) return rc;
  if (!vals) return fail(SE_ERR_ARG, "null host array");
  CK(cudaMemcpyAsync(vals, field->vals, sizeof(double) * field->mesh->nVertsTotal * field->ndofs,
                     cudaMemcpyDeviceToHost, g_stream));
  return SE_OK;
}
int se_field_device_ptr(se_field* field, double** dptr) {
  if (int rc = check_field(field)) return rc;
  if (!dptr) return fail(SE_ERR_ARG, "null argument");
  *dptr = field->vals;
  return SE_OK;
}
int se_field_copy(se_field* dst, const se_field* src) {
  if (int rc = check_field(dst)) return rc;
  if (int rc = check_field(src)) return rc;
  if (dst->mesh->nVertsTotal != src->mesh->nVertsTotal || dst->ndofs != src->ndofs)
    return fail(SE_ERR_ARG, "field shapes differ");
  if (dst == src) return SE_OK;
  CK(launch_copy(dst->vals, src->vals, (size_t)dst->mesh->nVertsTotal * dst->ndofs, g_stream));
  return SE_OK;
}
int se_field_periodic_update(se_field* field) {
  if (int rc = check_field(field)) return rc;
  CK(launch_periodic_update(field->mesh->dev, field->ndofs, field->vals, g_stream));
  return SE_OK;
}
int se_field_integrate(const se_field* field, int dof, int average, double* out) {
  if (int rc = check_field(field)) return rc;
  if (!out || dof < 0 || dof >= field->ndofs) return fail(SE_ERR_ARG, "bad argument");
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  CK(launch_quadrature(field->mesh->dev, field->ndofs, dof, field->vals, nullptr, g_scratch,
                       kScratch, g_scratch + kScratch, g_stream));
  double r[2];
  CK(cudaMemcpyAsync(r, g_scratch + kScratch, sizeof(r), cudaMemcpyDeviceToHost, g_stream));
  CK(cudaStreamSynchronize(g_stream));
  const MeshDev& m = field->mesh->dev;
  *out = average ? r[0] / ((m.max[0] - m.min[0]) * (m.max[1] - m.min[1])) : r[0];
  return SE_OK;
}
// Field::Save / Field::Read (src/base/Field.cpp:256-368) in raw binary:
// file "<name>.<time step, 5 digits>.seb" holding the HDF5 file's content
// in order: magic "SEFIELD1", dimensions (int32, 2), mesh resolution (int32
// nVerts[0]-1, nVerts[1]-1), rows (int64 nVertsTotal), columns (int32
// nDofs), then the /data dataset as double[rows][columns]; little-endian.
namespace {
const char kFieldMagic[8] = {'S', 'E', 'F', 'I', 'E', 'L', 'D', '1'};
std::string field_file(const char* name, int step) {
  char buf[32];
  snprintf(buf, sizeof(buf), ".%.5u.seb", (unsigned)step);
  return std::string(name) + buf;
}
}  // namespace

int se_field_save(const se_field* field, const char* name, int time_step) {
  if (int rc = check_field(field)) return rc;
  if (!name || time_step < 0) return fail(SE_ERR_ARG, "bad name or time step");
  const se_mesh* me = field->mesh;
  const size_t nv = (size_t)me->nVertsTotal, nd = (size_t)field->ndofs;
  std::vector<double> h(nv * nd);
  CK(cudaMemcpyAsync(h.data(), field->vals, sizeof(double) * h.size(), cudaMemcpyDeviceToHost,
                     g_stream));
  CK(cudaStreamSynchronize(g_stream));
  const std::string fn = field_file(name, time_step);
  FILE* f = std::fopen(fn.c_str(), "wb");
  if (!f) return fail(SE_ERR_ARG, "cannot create %s", fn.c_str());
  const int32_t dims = 2;
  const int32_t res[2] = {me->dev.nVerts[0] - 1, me->dev.nVerts[1] - 1};
  const int64_t rows = (int64_t)nv;
  const int32_t cols = (int32_t)nd;
  bool ok = std::fwrite(kFieldMagic, 1, 8, f) == 8 && std::fwrite(&dims, 4, 1, f) == 1 &&
            std::fwrite(res, 4, 2, f) == 2 && std::fwrite(&rows, 8, 1, f) == 1 &&
            std::fwrite(&cols, 4, 1, f) == 1 &&
            std::fwrite(h.data(), sizeof(double), h.size(), f) == h.size();
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) return fail(SE_ERR_ARG, "writing %s failed", fn.c_str());
  return SE_OK;
}

int se_field_read(se_field* field, const char* name, int time_step) {
  if (int rc = check_field(field)) return rc;
  if (!name || time_step < 0) return fail(SE_ERR_ARG, "bad name or time step");
  const se_mesh* me = field->mesh;
  const std::string fn = field_file(name, time_step);
  FILE* f = std::fopen(fn.c_str(), "rb");
  if (!f) return fail(SE_ERR_ARG, "cannot open %s", fn.c_str());
  char magic[8];
  int32_t dims = 0, res[2] = {0, 0}, cols = 0;
  int64_t rows = 0;
  bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, kFieldMagic, 8) == 0 &&
            std::fread(&dims, 4, 1, f) == 1 && std::fread(res, 4, 2, f) == 2 &&
            std::fread(&rows, 8, 1, f) == 1 && std::fread(&cols, 4, 1, f) == 1;
  if (!ok || dims != 2 || res[0] != me->dev.nVerts[0] - 1 || res[1] != me->dev.nVerts[1] - 1 ||
      rows != (int64_t)me->nVertsTotal || cols != field->ndofs) {
    std::fclose(f);
    return fail(SE_ERR_ARG, "%s does not hold a field of this mesh and size", fn.c_str());
  }
  std::vector<double> h((size_t)rows * cols);
  ok = std::fread(h.data(), sizeof(double), h.size(), f) == h.size();
  std::fclose(f);
  if (!ok) return fail(SE_ERR_ARG, "%s is truncated", fn.c_str());
  CK(cudaMemcpyAsync(field->vals, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice,
                     g_stream));
  CK(cudaStreamSynchronize(g_stream));
  return SE_OK;
}

// ------------------------------------------------------ mesh and XDMF ----
// Mesh::Save (src/base/Mesh.cpp:366-489) and the XDMF writers
// (src/base/Utils.cpp:53-229) with raw little-endian binary in place of
// HDF5. "<name>.seb" holds, in the HDF5 file's order: the magic "SEMESH01",
// the dimensions (int32 2, int32 pad), the mesh resolution (int32
// nVerts-1 per direction), /min and /max (double[2] each), the counts
// (int64 nVertsTotal, int64 linear quads), /vertices (double[nVertsTotal][2])
// and /connectivity (int32[quads][4], the reference's linear quads). The XDMF
// files reference these and the fields' ".seb" files as Binary DataItems
// with their byte offsets (Seek) past the headers.
namespace {
const char kMeshMagic[8] = {'S', 'E', 'M', 'E', 'S', 'H', '0', '1'};
constexpr long kMeshHeaderBytes = 72;
constexpr long kFieldHeaderBytes = 32;  // "SEFIELD1", dims, resolution, rows, columns
std::string step_tag(int step) {
  char buf[16];
  snprintf(buf, sizeof(buf), "%.5u", (unsigned)step);
  return buf;
}
// operator<< of a double on a default std::ostream (6 significant digits)
std::string fmt_double(double v) {
  char buf[64];
  snprintf(buf, sizeof(buf), "%g", v);
  return buf;
}
bool write_text(const std::string& fn, const std::string& text, const char* mode) {
  FILE* f = std::fopen(fn.c_str(), mode);
  if (!f) return false;
  const bool ok = std::fwrite(text.data(), 1, text.size(), f) == text.size();
  return (std::fclose(f) == 0) && ok;
}
const char* kXdmfHead =
    "<?xml version=\"1.0\" ?>\n<!DOCTYPE Xdmf SYSTEM \"Xdmf.dtd\" []>\n"
    "<Xdmf xmlns:xi=\"http://www.w3.org/2001/XInclude\" Version=\"2.0\">\n\n<Domain>\n\n";
const char* kXdmfFoot = "</Domain>\n\n</Xdmf>\n\n";
}  // namespace

int se_mesh_save(const se_mesh* mesh, const char* name) {
  if (!mesh || !name) return fail(SE_ERR_ARG, "null argument");
  const MeshDev& d = mesh->dev;
  const int64_t nv = mesh->nVertsTotal;
  const int32_t nl[2] = {d.nVerts[0] - 1, d.nVerts[1] - 1};
  const int64_t nq = (int64_t)nl[0] * nl[1];
  std::vector<double> verts(2 * (size_t)nv);
  if (int rc = se_mesh_verts(mesh, verts.data())) return rc;
  std::vector<int32_t> conn(4 * (size_t)nq);
  for (int64_t e = 0; e < nq; e++) {
    const int32_t j = (int32_t)(e / nl[0]);
    int32_t* c = conn.data() + 4 * e;
    c[0] = (int32_t)e + j;
    c[1] = c[0] + 1;
    c[2] = c[1] + d.nVerts[0];
    c[3] = c[2] - 1;
  }
  const std::string fn = std::string(name) + ".seb";
  FILE* f = std::fopen(fn.c_str(), "wb");
  if (!f) return fail(SE_ERR_ARG, "cannot create %s", fn.c_str());
  const int32_t dims[2] = {2, 0};
  bool ok = std::fwrite(kMeshMagic, 1, 8, f) == 8 && std::fwrite(dims, 4, 2, f) == 2 &&
            std::fwrite(nl, 4, 2, f) == 2 && std::fwrite(d.min, 8, 2, f) == 2 &&
            std::fwrite(d.max, 8, 2, f) == 2 && std::fwrite(&nv, 8, 1, f) == 1 &&
            std::fwrite(&nq, 8, 1, f) == 1 &&
            std::fwrite(verts.data(), sizeof(double), verts.size(), f) == verts.size() &&
            std::fwrite(conn.data(), sizeof(int32_t), conn.size(), f) == conn.size();
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) return fail(SE_ERR_ARG, "writing %s failed", fn.c_str());
  return SE_OK;
}

int se_write_xdmf_header(int time_step) {
  if (time_step < 0) return fail(SE_ERR_ARG, "bad time step");
  if (!write_text("XDMF." + step_tag(time_step) + ".xmf", kXdmfHead, "w"))
    return fail(SE_ERR_ARG, "cannot write the XDMF header");
  return SE_OK;
}
int se_write_xdmf_footer(int time_step) {
  if (time_step < 0) return fail(SE_ERR_ARG, "bad time step");
  if (!write_text("XDMF." + step_tag(time_step) + ".xmf", kXdmfFoot, "a"))
    return fail(SE_ERR_ARG, "cannot write the XDMF footer");
  return SE_OK;
}

int se_write_xdmf(const se_field* const* fields, const char* const* names, int nfields,
                  const char* mesh_name, int time_step, double time, double dt) {
  if (!fields || !names || nfields < 1 || !mesh_name || time_step < 0)
    return fail(SE_ERR_ARG, "bad argument");
  for (int i = 0; i < nfields; i++) {
    if (int rc = check_field(fields[i])) return rc;
    if (!names[i]) return fail(SE_ERR_ARG, "null field name");
    if (fields[i]->mesh != fields[0]->mesh) return fail(SE_ERR_ARG, "fields on different meshes");
  }
  const std::string ts = step_tag(time_step);
  if (!write_text("time." + ts + ".ts", "time step:\t" + std::to_string(time_step) + "\ttime:\t" +
                                             fmt_double(time) + "\tdt:\t" + fmt_double(dt) + "\n",
                  "w"))
    return fail(SE_ERR_ARG, "cannot write time.%s.ts", ts.c_str());
  for (int i = 0; i < nfields; i++)
    if (int rc = se_field_save(fields[i], names[i], time_step)) return rc;
  const MeshDev& d = fields[0]->mesh->dev;
  const long nv = fields[0]->mesh->nVertsTotal;
  const long nq = (long)(d.nVerts[0] - 1) * (d.nVerts[1] - 1);
  const std::string N = std::to_string(nv), M = mesh_name;
  const std::string fl = "NumberType=\"Float\" Precision=\"8\" Endian=\"Little\"";
  auto bin = [&](const std::string& dims, long seek, const std::string& file,
                 const std::string& type) {
    return "<DataItem Format=\"Binary\" " + type + " Seek=\"" + std::to_string(seek) +
           "\" Dimensions=\"" + dims + "\">" + file + "</DataItem>\n";
  };
  auto slab = [&](int col, int width, const std::string& file, long seek, const char* nm,
                  const std::string& ind) {
    std::string t = ind + "<DataItem ItemType=\"HyperSlab\" Dimensions=\"" + N + " 1\"" +
                    (nm ? std::string(" Name=\"") + nm + "\"" : "") + ">\n";
    t += ind + "   <DataItem Dimensions=\"3 2\" Format=\"XML\"> 0 " + std::to_string(col) +
         " 1 1 " + N + " 1 </DataItem>\n";
    t += ind + "   " + bin(N + " " + std::to_string(width), seek, file, fl);
    t += ind + "</DataItem>\n";
    return t;
  };
  std::string x;
  x += "   <Grid Name=\"FEM_Grid_" + M + "\">\n\n";
  x += "      <Time Value=\"" + fmt_double(time) + "\" />\n\n";
  x += "         <Topology Type=\"Quadrilateral\" NumberOfElements=\"" + std::to_string(nq) +
       "\"> \n";
  x += "            " +
       bin(std::to_string(nq) + " 4", kMeshHeaderBytes + 16 * nv, M + ".seb",
           "NumberType=\"Int\" Precision=\"4\" Endian=\"Little\"");
  x += "         </Topology>\n\n";
  x += "         <Geometry Type=\"XYZ\">\n";
  x += "            <DataItem ItemType=\"Function\"  Dimensions=\"" + N +
       " 3\" Function=\"JOIN($0, $1, 0*$1)\">\n";
  x += slab(0, 2, M + ".seb", kMeshHeaderBytes, "XCoords", "               ");
  x += slab(1, 2, M + ".seb", kMeshHeaderBytes, "YCoords", "               ");
  x += "            </DataItem>\n";
  x += "         </Geometry>\n\n";
  for (int i = 0; i < nfields; i++) {
    const std::string fn = std::string(names[i]) + "." + ts + ".seb";
    if (fields[i]->ndofs == 1) {
      x += std::string("         <Attribute Type=\"Scalar\" Center=\"Node\" Name=\"") + names[i] +
           "\">\n";
      x += slab(0, 1, fn, kFieldHeaderBytes, nullptr, "            ");
      x += "         </Attribute>\n\n";
    } else {
      x += std::string("         <Attribute Type=\"Vector\" Center=\"Node\" Name=\"") + names[i] +
           "\">\n";
      x += "            <DataItem ItemType=\"Function\"  Dimensions=\"" + N +
           " 3\" Function=\"JOIN($0, $1, 0*$1)\">\n";
      x += slab(0, 2, fn, kFieldHeaderBytes, "XValue", "               ");
      x += slab(1, 2, fn, kFieldHeaderBytes, "YValue", "               ");
      x += "            </DataItem>\n";
      x += "         </Attribute>\n\n";
    }
  }
  x += "   </Grid>\n\n";
  if (!write_text("XDMF." + ts + ".xmf", x, "a")) return fail(SE_ERR_ARG, "cannot append XDMF.%s.xmf", ts.c_str());
  return SE_OK;
}

int se_write_xdmf_temporal(int n_time_steps, int dump_every) {
  if (n_time_steps < 0 || dump_every < 1) return fail(SE_ERR_ARG, "bad step counts");
  const std::string inc =
      "   <xi:include href=\"XDMF.FilesField.xdmf\" xpointer=\"xpointer(//Xdmf/Grid)\"/>\n\n";
  const std::string body = std::string(kXdmfHead) + inc + kXdmfFoot;
  if (!write_text("XDMF.temporalAll.xmf", body, "w") ||
      !write_text("XDMF.temporalFields.xmf", body, "w"))
    return fail(SE_ERR_ARG, "cannot write the temporal XDMF files");
  std::string c =
      "<?xml version=\"1.0\" ?>\n<Xdmf xmlns:xi=\"http://www.w3.org/2001/XInclude\" "
      "Version=\"2.0\">\n<Grid GridType=\"Collection\" CollectionType=\"Temporal\" "
      "Name=\"FEM_Mesh_Fields\">\n";
  for (int s = 0; s <= n_time_steps; s += dump_every)
    c += "    <xi:include href=\"XDMF." + step_tag(s) +
         ".xmf\" xpointer=\"xpointer(//Xdmf/Domain/Grid[1])\"/>\n";
  c += "</Grid>\n</Xdmf>\n";
  if (!write_text("XDMF.FilesField.xdmf", c, "w"))
    return fail(SE_ERR_ARG, "cannot write XDMF.FilesField.xdmf");
  return SE_OK;
}

int se_field_gen_vel(const se_field* psi, se_field* vel) {
  if (int rc = check_field(psi)) return rc;
  if (int rc = check_field(vel)) return rc;
  if (psi->ndofs != 1 || vel->ndofs != 2) return fail(SE_ERR_ARG, "psi needs 1 and vel 2 components");
  if (psi->mesh != vel->mesh) return fail(SE_ERR_ARG, "psi and vel on different meshes");
  CK(launch_gen_vel(psi->mesh->dev, psi->vals, vel->vals, nullptr, g_stream));
  return SE_OK;
}
int se_field_interp_global(const se_field* field, const double* pts, int npts, double* out) {
  if (int rc = check_field(field)) return rc;
  if (npts < 0 || (npts && (!pts || !out))) return fail(SE_ERR_ARG, "bad argument");
  if (npts == 0) return SE_OK;
  double *dp = nullptr, *dout = nullptr;
  int rc;
  if ((rc = dalloc(&dp, 2 * (size_t)npts)) || (rc = dalloc(&dout, (size_t)npts * field->ndofs))) {
    dfree(dp);
    dfree(dout);
    return rc;
  }
  cudaStream_t s = g_stream;
  cudaError_t e = cudaMemcpyAsync(dp, pts, sizeof(double) * 2 * npts, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = launch_interp_global(field->mesh->dev, field->ndofs, field->vals, dp, npts, dout, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(out, dout, sizeof(double) * npts * field->ndofs, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  dfree(dp);
  dfree(dout);
  if (e != cudaSuccess) return cuda_fail(e, "interp_global");
  return SE_OK;
}

// ------------------------------------------------------------ advector ----
int se_advector_create(se_field* field, se_field* velocity, se_field* field_prev,
                       se_field* vel_prev, se_advector** out) {
  if (!out) return fail(SE_ERR_ARG, "null argument");
  *out = nullptr;
  if (int rc = check_field(field)) return rc;
  if (int rc = check_field(velocity)) return rc;
  if (velocity->ndofs != 2) return fail(SE_ERR_ARG, "velocity needs 2 components");
  if (velocity->mesh != field->mesh) return fail(SE_ERR_ARG, "velocity on another mesh");
  if ((field_prev == nullptr) != (vel_prev == nullptr))
    return fail(SE_ERR_ARG, "second order needs both previous fields");
  if (field_prev) {
    if (int rc = check_field(field_prev)) return rc;
    if (int rc = check_field(vel_prev)) return rc;
    if (field_prev->mesh != field->mesh || vel_prev->mesh != field->mesh ||
        field_prev->ndofs != field->ndofs || vel_prev->ndofs != 2)
      return fail(SE_ERR_ARG, "previous fields do not match");
  }
  if (field->mesh->dev.N < 3)
    return fail(SE_ERR_UNSUPPORTED, "N < 3 uses the reference's bicubic path, not built");
  se_advector* a = new se_advector();
  a->field = field;
  a->vel = velocity;
  a->field_prev = field_prev;
  a->vel_prev = vel_prev;
  int rc = dalloc(&a->err, 1);
  if (rc) {
    delete a;
    return rc;
  }
  if ((rc = se_field_create(field->mesh, field->ndofs, field->bcs, &a->sl))) {
    dfree(a->err);
    delete a;
    return rc;
  }
  // fieldSL starts as a copy of the field (src/base/Advector.cpp:63-64)
  if ((rc = se_field_copy(a->sl, field))) {
    se_field_destroy(a->sl);
    dfree(a->err);
    delete a;
    return rc;
  }
  *out = a;
  return SE_OK;
}
int se_advector_destroy(se_advector* adv) {
  if (!adv) return SE_OK;
  se_field_destroy(adv->sl);
  dfree(adv->dep_el);
  dfree(adv->dep_xy);
  dfree(adv->err);
  delete adv;
  return SE_OK;
}
int se_advect(se_advector* adv, double dt) {
  if (!adv) return fail(SE_ERR_ARG, "null advector");
  const se_mesh* me = adv->field->mesh;
  // the error word is read back only with the recorded departures: cleared
  // for the advections that record them
  if (adv->record) CK(cudaMemsetAsync(adv->err, 0, sizeof(unsigned), g_stream));
  CK(launch_sl(me->dev, adv->field->ndofs, adv->field->vals, adv->vel->vals,
               adv->field_prev ? adv->field_prev->vals : nullptr,
               adv->vel_prev ? adv->vel_prev->vals : nullptr, dt, adv->sl->vals,
               adv->record ? adv->dep_el : nullptr, adv->record ? adv->dep_xy : nullptr,
               adv->err, g_stream));
  return SE_OK;
}
int se_advector_field_sl(se_advector* adv, se_field** field_sl) {
  if (!adv || !field_sl) return fail(SE_ERR_ARG, "null argument");
  *field_sl = adv->sl;
  return SE_OK;
}
int se_advector_departures(se_advector* adv, int* el, double* xy) {
  if (!adv) return fail(SE_ERR_ARG, "null advector");
  const int nv = adv->field->mesh->nVertsTotal;
  const int k = adv->field_prev ? 2 : 1;
  if (!adv->record) {
    int rc;
    if ((rc = dalloc(&adv->dep_el, (size_t)k * nv)) || (rc = dalloc(&adv->dep_xy, (size_t)2 * k * nv)))
      return rc;
    adv->record = true;
    return fail(SE_ERR_ARG, "departure recording enabled; call se_advect first");
  }
  if (el) CK(cudaMemcpyAsync(el, adv->dep_el, sizeof(int) * k * nv, cudaMemcpyDeviceToHost, g_stream));
  if (xy)
    CK(cudaMemcpyAsync(xy, adv->dep_xy, sizeof(double) * 2 * k * nv, cudaMemcpyDeviceToHost,
                       g_stream));
  CK(cudaStreamSynchronize(g_stream));
  unsigned err = 0;
  CK(cudaMemcpy(&err, adv->err, sizeof(err), cudaMemcpyDeviceToHost));
  if (err & KERR_DOMAIN) return fail(SE_ERR_DOMAIN, "a departure point left the mesh");
  return SE_OK;
}

// -------------------------------------------------------------- linsys ----
int se_solver_opts_default(se_solver_opts* o) {
  if (!o) return fail(SE_ERR_ARG, "null options");
  o->rtol = 1e-5;
  o->atol = 1e-50;
  o->dtol = 1e5;
  o->max_it = 10000;
  o->norm_type = SE_NORM_PRECONDITIONED;
  o->mode = SE_MODE_REFERENCE;
  o->precision = SE_PREC_FP64;
  o->inner_max_it = 2000;
  o->inner_rtol = 1e-6;
  o->method = SE_METHOD_CG;
  return SE_OK;
}

int se_solver_opts_parse(se_solver_opts* o, const char* prefix, const char* options) {
  if (!o || !options) return fail(SE_ERR_ARG, "null argument");
  std::string pre = std::string("-") + (prefix ? prefix : "");
  std::vector<std::string> tok;
  {
    std::string cur;
    for (const char* p = options;; p++) {
      if (*p == 0 || *p == ' ' || *p == '\t' || *p == '\n') {
        if (!cur.empty()) tok.push_back(cur);
        cur.clear();
        if (*p == 0) break;
      } else {
        cur.push_back(*p);
      }
    }
  }
  for (size_t i = 0; i < tok.size(); i++) {
    const std::string& t = tok[i];
    if (t.compare(0, pre.size(), pre) != 0) continue;
    std::string key = t.substr(pre.size());
    std::string val = (i + 1 < tok.size() && tok[i + 1][0] != '-') ? tok[i + 1] : "";
    if (!val.empty()) i++;
    char* end = nullptr;
    if (key == "ksp_type") {
      if (val == "cg") o->method = SE_METHOD_CG;
      else if (val == "preonly") o->method = SE_METHOD_FDM;
      else return fail(SE_ERR_UNSUPPORTED, "ksp_type %s (cg, or preonly with pc_type fdm)", val.c_str());
    } else if (key == "pc_type") {
      if (val == "fdm") o->method = SE_METHOD_FDM;
      else if (val != "jacobi")
        return fail(SE_ERR_UNSUPPORTED, "pc_type %s (jacobi, or fdm)", val.c_str());
    } else if (key == "ksp_rtol") {
      o->rtol = std::strtod(val.c_str(), &end);
    } else if (key == "ksp_atol") {
      o->atol = std::strtod(val.c_str(), &end);
    } else if (key == "ksp_divtol") {
      o->dtol = std::strtod(val.c_str(), &end);
    } else if (key == "ksp_max_it") {
      o->max_it = (int)std::strtol(val.c_str(), &end, 10);
    } else if (key == "ksp_norm_type") {
      if (val == "preconditioned") o->norm_type = SE_NORM_PRECONDITIONED;
      else if (val == "unpreconditioned") o->norm_type = SE_NORM_UNPRECONDITIONED;
      else if (val == "natural") o->norm_type = SE_NORM_NATURAL;
      else return fail(SE_ERR_UNSUPPORTED, "ksp_norm_type %s", val.c_str());
    } else if (key == "precision") {
      // Not a PETSc key: the FDM solve's arithmetic (FP64, or the
      // reduced-precision inverses refined to the same FP64 tolerance).
      if (val == "fp64") o->precision = SE_PREC_FP64;
      else if (val == "mixed") o->precision = SE_PREC_MIXED;
      else if (val == "fp64_tc") o->precision = SE_PREC_FP64_TC;
      else if (val == "bf16") o->precision = SE_PREC_BF16;
      else if (val == "fp16") o->precision = SE_PREC_FP16;
      else return fail(SE_ERR_UNSUPPORTED, "precision %s (fp64, mixed, fp64_tc, bf16, fp16)", val.c_str());
    }
  }
  return SE_OK;
}

namespace {
// Solver options this library can run.
int check_opts(const se_solver_opts* o) {
  if (o->method != SE_METHOD_CG && o->method != SE_METHOD_FDM)
    return fail(SE_ERR_ARG, "unknown method %d", o->method);
  if (o->precision != SE_PREC_FP64 && o->precision != SE_PREC_MIXED && o->precision != SE_PREC_BF16 &&
      o->precision != SE_PREC_FP64_TC && o->precision != SE_PREC_FP16)
    return fail(SE_ERR_ARG, "unknown precision %d", o->precision);
  if (o->method == SE_METHOD_FDM && o->precision == SE_PREC_FP16)
    return fail(SE_ERR_UNSUPPORTED, "SE_PREC_FP16 with SE_METHOD_FDM (BF16, MIXED or FP64_TC)");
  if (o->method == SE_METHOD_CG && o->precision != SE_PREC_FP64 && o->precision != SE_PREC_BF16 &&
      o->precision != SE_PREC_FP16)
    return fail(SE_ERR_UNSUPPORTED, "SE_METHOD_CG runs in FP64, BF16 or FP16");
  if (o->norm_type < SE_NORM_PRECONDITIONED || o->norm_type > SE_NORM_NATURAL)
    return fail(SE_ERR_ARG, "unknown norm type %d", o->norm_type);
  if (o->mode != SE_MODE_REFERENCE && o->mode != SE_MODE_EXACT)
    return fail(SE_ERR_ARG, "unknown mode %d", o->mode);
  if (o->max_it < 0) return fail(SE_ERR_ARG, "negative max_it");
  return SE_OK;
}

int linsys_create(se_field* sol, se_field* rhs, bool poisson, double c, double nu, double dt,
                  int svv, const se_solver_opts* opts, se_linsys** out) {
  if (!out) return fail(SE_ERR_ARG, "null argument");
  *out = nullptr;
  if (opts)
    if (int rc = check_opts(opts)) return rc;
  if (int rc = check_field(sol)) return rc;
  if (sol->ndofs != 1) return fail(SE_ERR_UNSUPPORTED, "only scalar solution fields");
  if (rhs) {
    if (int rc = check_field(rhs)) return rc;
    if (rhs->mesh != sol->mesh || rhs->ndofs != 1) return fail(SE_ERR_ARG, "rhs does not match sol");
  }
  const MeshDev& m = sol->mesh->dev;
  for (int k = 0; k < 2; k++)
    if (m.periodic[k] && m.nEls[k] < 2)
      return fail(SE_ERR_UNSUPPORTED, "a periodic direction needs at least 2 elements");
  if (svv < 0 || svv > m.N) return fail(SE_ERR_ARG, "svvCutoff %d outside [0, N = %d]", svv, m.N);
  if (svv && opts && opts->method == SE_METHOD_FDM)
    return fail(SE_ERR_UNSUPPORTED, "the SVV operator needs SE_METHOD_CG (no fast diagonalization)");
  se_linsys* ls = new se_linsys();
  std::memset((void*)ls, 0, sizeof(*ls));
  ls->sol = sol;
  ls->rhs = rhs;
  ls->poisson = poisson;
  ls->c = c;
  ls->nu = nu;
  ls->dt = dt;
  ls->svv = svv;
  if (opts) ls->opts = *opts; else se_solver_opts_default(&ls->opts);
  if (!sol->bcs) {
    int rc = se_bcs_create(sol->mesh, 0, 0, 0, 0, &ls->own_bcs);
    if (rc) {
      delete ls;
      return rc;
    }
  }
  fill_op(ls);
  ls->n = ls->op.G[0] * ls->op.G[1];
  int rc = linsys_alloc(ls);
  if (rc) {
    linsys_free(ls);
    return rc;
  }
  *out = ls;
  return SE_OK;
}
}  // namespace

int se_helmholtz_create(se_field* sol, se_field* rhs, double c, double nu, double dt,
                        int svvCutoff, const se_solver_opts* opts, se_linsys** out) {
  return linsys_create(sol, rhs, false, c, nu, dt, svvCutoff, opts, out);
}
int se_poisson_create(se_field* sol, se_field* rhs, double c, const se_solver_opts* opts,
                      se_linsys** out) {
  return linsys_create(sol, rhs, true, c, 0.0, 0.0, 0, opts, out);
}
int se_linsys_destroy(se_linsys* ls) {
  if (ls) linsys_free(ls);
  return SE_OK;
}
int se_linsys_set_opts(se_linsys* ls, const se_solver_opts* opts) {
  if (!ls || !opts) return fail(SE_ERR_ARG, "null argument");
  if (int rc = check_opts(opts)) return rc;
  if (ls->svv && opts->method == SE_METHOD_FDM)
    return fail(SE_ERR_UNSUPPORTED, "the SVV operator needs SE_METHOD_CG (no fast diagonalization)");
  int old_mode = ls->opts.mode;
  ls->opts = *opts;
  if (opts->mode != old_mode) {
    fill_op(ls);
    ls->assembled = false;
    if (ls->X1) {  // the FDM's Jacobi inverse follows the operator
      CK(launch_op_diag(ls->op, ls->dinv, g_stream));
      CK(launch_invert(ls->dinv, ls->n, g_stream));
    }
  }
  return SE_OK;
}
int se_linsys_assemble(se_linsys* ls) {
  if (!ls) return fail(SE_ERR_ARG, "null system");
  CK(launch_lift(ls->op, ls->sol->mesh->dev, ls->sol->vals, ls->lift, g_stream));
  ls->assembled = true;
  return SE_OK;
}
int se_linsys_solve(se_linsys* ls, int remove_null_space, se_solve_stats* stats) {
  if (!ls) return fail(SE_ERR_ARG, "null system");
  if (remove_null_space < 0 || remove_null_space > 2)
    return fail(SE_ERR_ARG, "remove_null_space must be 0, 1 or 2");
  if (!ls->assembled)
    if (int rc = se_linsys_assemble(ls)) return rc;
  const MeshDev& m = ls->sol->mesh->dev;
  CgSolve st;
  float kms = 0.f;
  int rc, outer = 0;
  if (ls->opts.method == SE_METHOD_FDM) {
    // right-hand side assembly and field update are inside the FDM graph
    rc = run_fdm(ls, remove_null_space, &st, &kms);
    if (rc) return rc;
  } else {
    CK(launch_rhs_assemble(ls->op, m, ls->rhs ? ls->rhs->vals : nullptr, ls->lift, ls->f, g_stream));
    if (ls->opts.precision == SE_PREC_FP64) {
      rc = run_cg(ls, ls->f, ls->x, ls->opts.rtol, ls->opts.atol, ls->opts.dtol, ls->opts.max_it,
                  remove_null_space, &st, &kms);
    } else {
      if (remove_null_space)
        return fail(SE_ERR_UNSUPPORTED, "the reduced-precision CG does not remove a null space");
      rc = run_mixed_cg(ls, ls->opts.precision == SE_PREC_BF16 ? 1 : 2, &st, &outer, &kms);
    }
    if (rc) return rc;
    CK(launch_update_field(ls->op, m, ls->x, ls->sol->vals, g_stream));
  }
  if (stats) {
    stats->reason = st.reason;
    stats->its = st.its;
    stats->outer_its = ls->opts.method == SE_METHOD_FDM ? st.its : outer;
    stats->rnorm = st.dp;
    stats->rnorm0 = st.rnorm0;
    stats->kernel_ms = kms;
  }
  if (st.reason < 0) return fail(SE_ERR_NOT_CONVERGED, "KSP diverged, reason %d after %d its",
                                 st.reason, st.its);
  return SE_OK;
}
int se_linsys_solve_batch(se_linsys** systems, int n, int remove_null_space, se_solve_stats* stats) {
  if (!systems || n < 0) return fail(SE_ERR_ARG, "bad argument");
  if (remove_null_space < 0 || remove_null_space > 2)
    return fail(SE_ERR_ARG, "remove_null_space must be 0, 1 or 2");
  for (int i = 0; i < n; i++)
    if (!systems[i]) return fail(SE_ERR_ARG, "null system %d", i);
  for (int i = 0; i < n; i++)
    if (!systems[i]->assembled)
      if (int rc = se_linsys_assemble(systems[i])) return rc;
  std::vector<CgSolve> st(n);
  std::vector<float> kms(n, 0.f);
  // fast-diagonalization solves: graphs overlapped over a pool of streams
  static thread_local std::vector<cudaStream_t> pool;
  if (pool.empty()) {
    for (int k = 0; k < 8; k++) {
      cudaStream_t s;
      CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
      pool.push_back(s);
    }
  }
  const cudaStream_t saved = g_stream;
  cudaEvent_t ready;
  CK(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
  CK(cudaEventRecord(ready, saved));
  std::vector<int> fdm_idx, mixed_idx;
  std::map<int, std::vector<int>> cg_groups;
  for (int i = 0; i < n; i++) {
    if (systems[i]->opts.method == SE_METHOD_FDM) fdm_idx.push_back(i);
    else if (systems[i]->opts.precision != SE_PREC_FP64) mixed_idx.push_back(i);  // one by one
    else cg_groups[systems[i]->op.d[0].N].push_back(i);
  }
  std::vector<se_solve_stats> mixed_stats(mixed_idx.size());
  int rc = SE_OK;
  for (size_t k = 0; k < fdm_idx.size() && !rc; k++) {
    g_stream = pool[k % pool.size()];
    if (k < pool.size()) cudaStreamWaitEvent(g_stream, ready, 0);
    rc = fdm_launch(systems[fdm_idx[k]], remove_null_space, true);
  }
  g_stream = saved;
  for (auto& grp : cg_groups) {
    if (rc) break;
    std::vector<int>& idx = grp.second;
    for (size_t off = 0; off < idx.size() && !rc; off += 256) {
      std::vector<se_linsys*> sys;
      for (size_t j = off; j < std::min(idx.size(), off + 256); j++) {
        se_linsys* ls = systems[idx[j]];
        const MeshDev& m = ls->sol->mesh->dev;
        CK(launch_rhs_assemble(ls->op, m, ls->rhs ? ls->rhs->vals : nullptr, ls->lift, ls->f, g_stream));
        sys.push_back(ls);
      }
      std::vector<CgSolve> out;
      float t = 0.f;
      rc = solve_cg_group(sys, remove_null_space, out, &t);
      for (size_t j = 0; j < sys.size() && !rc; j++) {
        st[idx[off + j]] = out[j];
        kms[idx[off + j]] = t;
        const MeshDev& m = sys[j]->sol->mesh->dev;
        if (launch_update_field(sys[j]->op, m, sys[j]->x, sys[j]->sol->vals, g_stream) != cudaSuccess)
          rc = fail(SE_ERR_CUDA, "field update");
      }
    }
  }
  for (size_t k = 0; k < mixed_idx.size() && !rc; k++) {
    rc = se_linsys_solve(systems[mixed_idx[k]], remove_null_space, &mixed_stats[k]);
    if (rc == SE_ERR_NOT_CONVERGED) rc = SE_OK;  // reported with the others below
  }
  for (size_t k = 0; k < fdm_idx.size() && !rc; k++)
    rc = fdm_finish(systems[fdm_idx[k]], &st[fdm_idx[k]], &kms[fdm_idx[k]]);
  // the caller's stream sees every solve's result
  for (size_t k = 0; k < pool.size() && k < fdm_idx.size(); k++) {
    cudaEvent_t done;
    if (cudaEventCreateWithFlags(&done, cudaEventDisableTiming) == cudaSuccess) {
      cudaEventRecord(done, pool[k]);
      cudaStreamWaitEvent(saved, done, 0);
      cudaEventDestroy(done);
    }
  }
  cudaEventDestroy(ready);
  if (rc) return rc;
  int worst = SE_OK;
  std::vector<int> mixed_at(n, -1);
  for (size_t k = 0; k < mixed_idx.size(); k++) mixed_at[mixed_idx[k]] = (int)k;
  for (int i = 0; i < n; i++) {
    if (mixed_at[i] >= 0) {
      const se_solve_stats& ms = mixed_stats[mixed_at[i]];
      if (stats) stats[i] = ms;
      if (ms.reason < 0) worst = SE_ERR_NOT_CONVERGED;
      continue;
    }
    if (stats) {
      se_solve_stats& o = stats[i];
      o.reason = st[i].reason;
      o.its = st[i].its;
      o.outer_its = systems[i]->opts.method == SE_METHOD_FDM ? st[i].its : 0;
      o.rnorm = st[i].dp;
      o.rnorm0 = st[i].rnorm0;
      o.kernel_ms = kms[i];
    }
    if (st[i].reason < 0) worst = SE_ERR_NOT_CONVERGED;
  }
  if (worst) return fail(worst, "at least one system did not converge");
  return SE_OK;
}
int se_linsys_solve_async(se_linsys* ls, int remove_null_space) {
  if (!ls) return fail(SE_ERR_ARG, "null system");
  if (remove_null_space < 0 || remove_null_space > 2)
    return fail(SE_ERR_ARG, "remove_null_space must be 0, 1 or 2");
  if (!ls->assembled)
    if (int rc = se_linsys_assemble(ls)) return rc;
  if (ls->opts.method != SE_METHOD_FDM) {
    // the CG path reads its state back on the host: solve now, keep the stats
    ls->async_rc = se_linsys_solve(ls, remove_null_space, &ls->async_stats);
    ls->async_pending = 2;
    return ls->async_rc == SE_ERR_NOT_CONVERGED ? SE_OK : ls->async_rc;
  }
  if (int rc = fdm_launch(ls, remove_null_space, false)) return rc;
  ls->async_pending = 1;
  return SE_OK;
}
int se_linsys_solve_finish(se_linsys* ls, se_solve_stats* stats) {
  if (!ls || !ls->async_pending) return fail(SE_ERR_ARG, "no solve queued");
  if (ls->async_pending == 2) {
    ls->async_pending = 0;
    if (stats) *stats = ls->async_stats;
    return ls->async_rc;
  }
  ls->async_pending = 0;
  CgSolve st;
  float kms = 0.f;
  if (int rc = fdm_finish(ls, &st, &kms)) return rc;
  if (stats) {
    stats->reason = st.reason;
    stats->its = st.its;
    stats->outer_its = st.its;
    stats->rnorm = st.dp;
    stats->rnorm0 = st.rnorm0;
    stats->kernel_ms = kms;
  }
  if (st.reason < 0) return fail(SE_ERR_NOT_CONVERGED, "KSP diverged, reason %d after %d its",
                                 st.reason, st.its);
  return SE_OK;
}
int se_linsys_apply(se_linsys* ls, const double* x_dev, double* y_dev) {
  if (!ls || !x_dev || !y_dev) return fail(SE_ERR_ARG, "null argument");
  // orders 4 to 8 (and SVV systems) run kernels without barrier waits;
  // the TMA-staged kernel of the other orders reports a barrier that timed
  // out in the error word, read back here
  const int N = ls->op.d[0].N;
  const bool waits = ls->op.gamma == 0.0 && (N < 4 || N > 8);
  if (waits) CK(cudaMemsetAsync(ls->d_err, 0, sizeof(unsigned), g_stream));
  CK(launch_op_apply(ls->op, x_dev, y_dev, ls->d_err, g_stream));
  if (waits) {
    unsigned err = 0;
    CK(cudaMemcpyAsync(&err, ls->d_err, sizeof(unsigned), cudaMemcpyDeviceToHost, g_stream));
    CK(cudaStreamSynchronize(g_stream));
    if (err & KERR_BARRIER_TIMEOUT) return fail(SE_ERR_TIMEOUT, "apply: a TMA stage never arrived");
  }
  return SE_OK;
}
int se_linsys_fdm_apply(se_linsys* ls, const double* r_dev, double* x_dev) {
  if (!ls || !r_dev || !x_dev) return fail(SE_ERR_ARG, "null argument");
  if (r_dev == x_dev) return fail(SE_ERR_ARG, "r and x must not alias");
  if (int rc = fdm_setup(ls, 0)) return rc;
  return fdm_apply64(ls, r_dev, x_dev, false);
}
int se_linsys_residual(se_linsys* ls, const double* x_dev, const double* b_dev, double* r_dev) {
  if (!ls || !x_dev || !b_dev || !r_dev) return fail(SE_ERR_ARG, "null argument");
  if (r_dev == x_dev || r_dev == b_dev) return fail(SE_ERR_ARG, "r must not alias x or b");
  if (!ls->fpart) {
    ls->fpart_n = std::max(kFdmPartials, std::max(residual_blocks(ls->op), residual_partial_blocks(ls->op)));
    if (int rc = dalloc(&ls->fpart, 2 * (size_t)ls->fpart_n + 16)) return rc;
  }
  CK(launch_residual(ls->op, x_dev, b_dev, r_dev, nullptr, 0, ls->fpart, g_stream));
  return SE_OK;
}
int se_linsys_fdm_apply_prec(se_linsys* ls, int precision, const double* r_dev, double* x_dev) {
  if (!ls || !r_dev || !x_dev) return fail(SE_ERR_ARG, "null argument");
  if (r_dev == x_dev) return fail(SE_ERR_ARG, "r and x must not alias");
  if (precision == SE_PREC_FP64) return se_linsys_fdm_apply(ls, r_dev, x_dev);
  if (precision != SE_PREC_MIXED)
    return fail(SE_ERR_UNSUPPORTED, "precision must be SE_PREC_FP64 or SE_PREC_MIXED");
  if (int rc = fdm_setup(ls, 1)) return rc;
  if (!ls->d_fparams) {  // the products report through the loop state's error word
    int rc;
    if ((rc = dalloc(&ls->d_fparams, 1)) || (rc = dalloc(&ls->d_fstate, 1)) ||
        (rc = dalloc(&ls->d_rescount, 1)))
      return rc;
    CK(cudaMemsetAsync(ls->d_rescount, 0, sizeof(unsigned), g_stream));
    CK(cudaMemsetAsync(ls->d_fstate, 0, sizeof(FdmState), g_stream));
  }
  CK(cudaMemsetAsync(x_dev, 0, sizeof(double) * ls->n, g_stream));
  return fdm_apply_tc(ls, r_dev, x_dev);
}
int se_linsys_apply_low(se_linsys* ls, int precision, const void* x_dev, float* y_dev) {
  if (!ls || !x_dev || !y_dev) return fail(SE_ERR_ARG, "null argument");
  if (precision != SE_PREC_BF16 && precision != SE_PREC_FP16)
    return fail(SE_ERR_ARG, "precision must be SE_PREC_BF16 or SE_PREC_FP16");
  if (ls->svv) return fail(SE_ERR_UNSUPPORTED, "the low-precision apply has no SVV term");
  CK(launch_op_apply_low(ls->op, precision == SE_PREC_FP16, x_dev, y_dev, g_stream));
  return SE_OK;
}
int se_linsys_diagonal(se_linsys* ls, double* d_dev) {
  if (!ls || !d_dev) return fail(SE_ERR_ARG, "null argument");
  CK(launch_op_diag(ls->op, d_dev, g_stream));
  return SE_OK;
}
int se_linsys_vec_size(const se_linsys* ls, int* n) {
  if (!ls || !n) return fail(SE_ERR_ARG, "null argument");
  *n = ls->n;
  return SE_OK;
}

// ----------------------------------------------------------- utilities ----
int se_calc_time_step(const se_field* velocity, double courant, double* dt) {
  if (int rc = check_field(velocity)) return rc;
  if (velocity->ndofs != 2 || !dt) return fail(SE_ERR_ARG, "bad argument");
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  CK(launch_max_speed_sq(velocity->mesh->nVertsTotal, velocity->vals, g_scratch, kScratch,
                         g_scratch + kScratch, g_stream));
  double mx = 0.0;
  CK(cudaMemcpyAsync(&mx, g_scratch + kScratch, sizeof(double), cudaMemcpyDeviceToHost, g_stream));
  CK(cudaStreamSynchronize(g_stream));
  const MeshDev& m = velocity->mesh->dev;
  double minSep = m.dx[0] < m.dx[1] ? m.dx[0] : m.dx[1];
  *dt = courant * minSep / std::sqrt(mx);
  return SE_OK;
}
int se_field_error(const se_field* numeric, const se_field* analytic, int dof, int normalise,
                   double* err) {
  if (int rc = check_field(numeric)) return rc;
  if (int rc = check_field(analytic)) return rc;
  if (!err || dof < 0 || dof >= numeric->ndofs || numeric->mesh != analytic->mesh ||
      numeric->ndofs != analytic->ndofs)
    return fail(SE_ERR_ARG, "bad argument");
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  CK(launch_quadrature(numeric->mesh->dev, numeric->ndofs, dof, numeric->vals, analytic->vals,
                       g_scratch, kScratch, g_scratch + kScratch, g_stream));
  double r[2];
  CK(cudaMemcpyAsync(r, g_scratch + kScratch, sizeof(r), cudaMemcpyDeviceToHost, g_stream));
  CK(cudaStreamSynchronize(g_stream));
  *err = normalise ? std::sqrt(r[0] / r[1]) : std::sqrt(r[0]);
  return SE_OK;
}

}  // extern "C"

// ===================================================== no-allocation solve ==
// se_helmholtz_solve_noalloc: the whole HelmholtzEqn/PoissonEqn
// construct-assemble-solve sequence in one call that allocates nothing. It
// is for callers that cannot call cudaMalloc: a model driver that reserves
// its whole device-memory budget at start-up (other components share the
// GPU and a later allocation may fail or evict them), or a time loop that
// cannot afford the implicit device-wide synchronisation cudaMalloc/cudaFree
// may cause in the middle of a step. The caller passes the field arrays;
// every temporary lives in g_noalloc_scratch below.
//
// Limits and sharing: at most kNoAllocMaxUnknowns vector unknowns and
// kNoAllocMaxTiles tiles of 32x16 unknowns per solve; larger systems are
// rejected with SE_ERR_UNSUPPORTED. Only the drop-in solver runs here
// (SE_METHOD_CG in SE_PREC_FP64); other methods and precisions are refused
// with SE_ERR_UNSUPPORTED. The array is held by every GPU that loads the
// library until the process exits, and every call on a device shares it and
// leaves its contents behind. Two calls whose device work overlapped would
// race on it, so each call holds g_noalloc_mu until its stream has finished
// its work. The first call on each device looks up the array's device address
// (cudaGetSymbolAddress, with that device current); make that first call
// before any stream capture.
namespace {
constexpr int kNoAllocMaxUnknowns = 65536;
constexpr int kNoAllocMaxTiles = 8192;
constexpr int kNoAllocMaxGrid = 4096;
constexpr size_t kNoAllocVecDoubles = 9 * (size_t)kNoAllocMaxUnknowns;  // f lift x r z p0 p1 w dinv
constexpr size_t kNoAllocPartialDoubles = 8 * (size_t)kNoAllocMaxGrid;  // two buffers
constexpr size_t kNoAllocSolveDoubles = (sizeof(CgSolve) + 255) / 256 * 256 / sizeof(double);
constexpr size_t kNoAllocTileDoubles = (sizeof(CgTile) * kNoAllocMaxTiles + 255) / 256 * 256 / sizeof(double);
constexpr size_t kNoAllocBeginDoubles = (sizeof(int) * (kNoAllocMaxGrid + 1) + 255) / 256 * 256 / sizeof(double);
// barrier count, generation, active count and error word, each on its own
// 128-byte line: 128 unsigned words
constexpr size_t kNoAllocWordDoubles = 64;
constexpr size_t kNoAllocDoubles = kNoAllocVecDoubles + kNoAllocPartialDoubles + kNoAllocSolveDoubles +
                                   kNoAllocTileDoubles + kNoAllocBeginDoubles + kNoAllocWordDoubles;
}  // namespace

// About 5 MB per device: 9 vectors of 65536 doubles plus the schedule.
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocDoubles];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;                // guards the host-side tables below
double* g_noalloc_dev[kMaxDevices];     // device address of the scratch, per device
CgTile g_noalloc_tiles[kNoAllocMaxTiles];
int g_noalloc_begin[kNoAllocMaxGrid + 1];
}  // namespace

extern "C" int se_helmholtz_solve_noalloc(const int nEls[2], int N, const double min[2],
                                          const double max[2], const int periodic[2],
                                          const int bcs[4], double c, double nu, double dt,
                                          int poisson, const se_solver_opts* opts,
                                          int remove_null_space, const double* rhs_dev,
                                          double* sol_dev, se_solve_stats* stats) {
  if (!nEls || !min || !max || !periodic || !bcs || !sol_dev)
    return fail(SE_ERR_ARG, "null argument");
  if (N < 2 || N > SE_MAXN)
    return fail(SE_ERR_UNSUPPORTED, "polynomial order %d outside [2, %d]", N, SE_MAXN);
  if (nEls[0] < 1 || nEls[1] < 1) return fail(SE_ERR_ARG, "element counts must be positive");
  if (!(max[0] > min[0]) || !(max[1] > min[1])) return fail(SE_ERR_ARG, "empty domain");
  if (remove_null_space < 0 || remove_null_space > 2)
    return fail(SE_ERR_ARG, "remove_null_space must be 0, 1 or 2");
  const bool b = bcs[0] != 0, t = bcs[1] != 0, l = bcs[2] != 0, r = bcs[3] != 0;
  const int perx = periodic[0] != 0, pery = periodic[1] != 0;
  if ((b || t) && pery) return fail(SE_ERR_ARG, "both periodic and non-periodic conditions in y");
  if ((l || r) && perx) return fail(SE_ERR_ARG, "both periodic and non-periodic conditions in x");
  if (pery && !perx) return fail(SE_ERR_UNSUPPORTED, "periodic in y only is not built by the reference");
  if (perx && !pery && b && !t)
    return fail(SE_ERR_UNSUPPORTED, "periodic x with a bottom wall only (reference: bc error)");
  if ((perx && nEls[0] < 2) || (pery && nEls[1] < 2))
    return fail(SE_ERR_UNSUPPORTED, "a periodic direction needs at least 2 elements");
  // the vertex grid must fit an int before any index is formed from it
  const long nvx = (long)nEls[0] * N + 1, nvy = (long)nEls[1] * N + 1;
  if (nvx * nvy > (1L << 30)) return fail(SE_ERR_UNSUPPORTED, "mesh too large");
  se_solver_opts o;
  if (opts) o = *opts; else se_solver_opts_default(&o);
  if (int rc = check_opts(&o)) return rc;
  // this entry point runs the drop-in solver only: Jacobi CG in FP64
  if (o.method != SE_METHOD_CG)
    return fail(SE_ERR_UNSUPPORTED, "the no-allocation solve runs SE_METHOD_CG only");
  if (o.precision != SE_PREC_FP64)
    return fail(SE_ERR_UNSUPPORTED, "the no-allocation solve runs SE_PREC_FP64 only");

  // host tables on the stack: mesh, boundary ranges, operator
  se_mesh mesh;
  gll_build(N, mesh.gll);
  MeshDev& md = mesh.dev;
  std::memset(&md, 0, sizeof(md));
  md.N = N;
  for (int k = 0; k < 2; k++) {
    md.nEls[k] = nEls[k];
    md.nVerts[k] = nEls[k] * N + 1;
    md.periodic[k] = k == 0 ? perx : pery;
    md.min[k] = min[k];
    md.max[k] = max[k];
    md.dx[k] = (md.max[k] - md.min[k]) / md.nEls[k];
    md.two_over_dx[k] = 2.0 / md.dx[k];
    md.span[k] = md.max[k] - md.min[k];
    md.nspan[k] = md.min[k] - md.max[k];
  }
  for (int i = 0; i <= N; i++) {
    md.abcissa[i] = mesh.gll.x[i];
    md.lambda[i] = mesh.gll.lambda[i];
    md.w[i] = mesh.gll.w[i];
  }
  OpDev op;
  std::memset(&op, 0, sizeof(op));
  op.d[0] = make_dir(md, 0, l, r);
  op.d[1] = make_dir(md, 1, b, t || pery);
  op.G[0] = op.d[0].hi - op.d[0].lo;
  op.G[1] = op.d[1].hi - op.d[1].lo;
  const long n = (long)op.G[0] * op.G[1];
  if (n <= 0) return fail(SE_ERR_ARG, "the system has no unknowns");
  if (n > kNoAllocMaxUnknowns)
    return fail(SE_ERR_UNSUPPORTED,
                "%ld unknowns exceed the no-allocation limit of %d; use se_helmholtz_create", n,
                kNoAllocMaxUnknowns);
  const long ntiles = (long)((op.G[0] + kCgTileX - 1) / kCgTileX) * ((op.G[1] + kCgTileY - 1) / kCgTileY);
  if (ntiles > kNoAllocMaxTiles)
    return fail(SE_ERR_UNSUPPORTED, "%ld tiles exceed the no-allocation limit of %d", ntiles,
                kNoAllocMaxTiles);
  const double hx = md.dx[0], hy = md.dx[1];
  const double s = poisson ? c : nu * dt;
  op.alpha = (poisson ? 0.0 : c) * (0.5 * hx) * (0.5 * hy);
  if (o.mode == SE_MODE_EXACT) {
    op.beta[0] = s * (hy / hx);
    op.beta[1] = s * (hx / hy);
  } else {
    op.beta[0] = s * (2.0 / hx) * (2.0 / hx);
    op.beta[1] = s * (2.0 / hy) * (2.0 / hy);
  }
  for (int a = 0; a < (N + 1) * (N + 1); a++) op.Kh[a] = mesh.gll.Kh[a];
  for (int a = 0; a <= N; a++) op.w[a] = mesh.gll.w[a];

  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return fail(SE_ERR_UNSUPPORTED, "device index %d", dev);
  if (!g_noalloc_dev[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
    g_noalloc_dev[dev] = static_cast<double*>(p);
  }
  double* base = g_noalloc_dev[dev];
  const size_t vn = kNoAllocMaxUnknowns;
  double *f = base, *lift = base + vn, *x = base + 2 * vn, *rr = base + 3 * vn, *z = base + 4 * vn,
         *p0 = base + 5 * vn, *p1 = base + 6 * vn, *w = base + 7 * vn, *dinv = base + 8 * vn;
  double* partials = base + kNoAllocVecDoubles;
  CgSolve* d_solve = reinterpret_cast<CgSolve*>(partials + kNoAllocPartialDoubles);
  CgTile* d_tiles = reinterpret_cast<CgTile*>(partials + kNoAllocPartialDoubles + kNoAllocSolveDoubles);
  int* d_begin = reinterpret_cast<int*>(partials + kNoAllocPartialDoubles + kNoAllocSolveDoubles +
                                        kNoAllocTileDoubles);
  unsigned* words = reinterpret_cast<unsigned*>(partials + kNoAllocPartialDoubles + kNoAllocSolveDoubles +
                                                kNoAllocTileDoubles + kNoAllocBeginDoubles);

  // schedule: same tile order, mode and contiguous block chunks as the
  // allocating path
  bool resident = false;
  const int maxg = std::min(cg_plan(dev, N, ntiles, 1, &resident), kNoAllocMaxGrid);
  if (maxg <= 0) return fail(SE_ERR_CUDA, "cannot size the cooperative CG launch");
  int nt = 0;
  for (int y = 0; y < op.G[1]; y += kCgTileY)
    for (int xx = 0; xx < op.G[0]; xx += kCgTileX) g_noalloc_tiles[nt++] = {0, xx, y, 0};
  const int grid = std::max(1, std::min(maxg, nt));
  for (int k = 0; k <= grid; k++) g_noalloc_begin[k] = (int)((long)nt * k / grid);
  for (int k = 0; k < grid; k++)
    for (int q = g_noalloc_begin[k]; q < g_noalloc_begin[k + 1]; q++) g_noalloc_tiles[q].seg = k;

  CgSolve cs;
  std::memset(&cs, 0, sizeof(cs));
  cs.op = op;
  cs.b = f;
  cs.x = x;
  cs.r = rr;
  cs.z = z;
  cs.p0 = p0;
  cs.p1 = p1;
  cs.w = w;
  cs.dinv = dinv;
  cs.rtol = o.rtol;
  cs.atol = o.atol;
  cs.dtol = o.dtol;
  cs.max_it = o.max_it;
  cs.norm_type = o.norm_type;
  cs.remove_null = remove_null_space;
  cs.n = (int)n;
  cs.seg_begin = 0;
  cs.seg_end = grid;

  cudaStream_t st = g_stream;
  // what must start at zero: the barrier words, the active count, the error word
  CK(cudaMemsetAsync(words, 0, sizeof(double) * kNoAllocWordDoubles, st));
  CK(cudaMemcpyAsync(d_tiles, g_noalloc_tiles, sizeof(CgTile) * nt, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(d_begin, g_noalloc_begin, sizeof(int) * (grid + 1), cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(d_solve, &cs, sizeof(cs), cudaMemcpyHostToDevice, st));
  CK(launch_lift(op, md, sol_dev, lift, st));
  CK(launch_rhs_assemble(op, md, rhs_dev, lift, f, st));
  CgBatch B;
  B.solves = d_solve;
  B.nsolves = 1;
  B.tiles = d_tiles;
  B.block_tile_begin = d_begin;
  B.partials = partials;
  B.nseg = grid;
  B.bar_count = words;
  B.bar_gen = words + 32;   // another 128-byte line
  B.n_active = reinterpret_cast<int*>(words + 64);
  B.err = words + 96;
  CK(launch_cg(B, grid, N, resident, st));
  CgSolve out;
  unsigned err = 0;
  CK(cudaMemcpyAsync(&out, d_solve, sizeof(out), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(&err, B.err, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
  CK(launch_update_field(op, md, x, sol_dev, st));
  CK(cudaStreamSynchronize(st));
  if (err & KERR_BARRIER_TIMEOUT) return fail(SE_ERR_TIMEOUT, "CG grid barrier timed out");
  if (stats) {
    stats->reason = out.reason;
    stats->its = out.its;
    stats->outer_its = 0;
    stats->rnorm = out.dp;
    stats->rnorm0 = out.rnorm0;
    stats->kernel_ms = 0.0;
  }
  if (out.reason < 0)
    return fail(SE_ERR_NOT_CONVERGED, "KSP diverged, reason %d after %d its", out.reason, out.its);
  return SE_OK;
}

// ------------------------------------------------------ two-layer QG step --
// TwoLayerQGEqn (src/qg/TwoLayerQGEqn.cpp:17-433) composed from this
// library's objects: GenPV, GenVel and the step's pointwise combinations as
// kernels (sl.cu), the PV advection by the SL advectors, the baroclinic
// Helmholtz and barotropic Poisson inversions by se_linsys (the method and
// precision of the given options), and SolveQ with its DissipationRHS as one
// kernel per layer. The reference's choices are kept: the first-order step
// applies SolveQ to layer 1 only; both layers' dissipation uses the first
// baroclinic solution tau1; the PV mass matrix is scaled by 1.5 from the
// first second-order step on.
struct se_qg2 {
  se_field *psi1, *omega1, *psi2, *omega2, *tau_e;  // the caller's
  double F1, F2, beta, E2, r, nu, dt;
  double a_mass;
  bool second_assembled;
  se_field *tau1, *chi1, *tau2, *chi2;              // psi1's boundary conditions
  se_field *psi1h, *psi2h, *om1h, *om2h;            // psi1's boundary conditions
  se_field *alpha1, *alpha2, *alpha1h, *alpha2h;    // psi1's boundary conditions
  se_field *alpha1p, *alpha2p;                      // no boundary conditions
  se_field *hrhs1, *frhs1, *hrhs2, *frhs2;          // no boundary conditions
  se_field *vel1, *vel2, *vel1p, *vel2p, *grad;     // 2 components
  se_field *tmp[4];
  se_linsys *helm1, *helm2, *fish1, *fish2;
  se_advector *adv1, *adv2, *adv1s, *adv2s;
  int nc;  // solves of the current step that did not converge
};

namespace {
int qg_release(se_qg2* q) {
  se_field** fs[] = {&q->tau1, &q->chi1, &q->tau2, &q->chi2, &q->psi1h, &q->psi2h, &q->om1h,
                     &q->om2h, &q->alpha1, &q->alpha2, &q->alpha1h, &q->alpha2h, &q->alpha1p,
                     &q->alpha2p, &q->hrhs1, &q->frhs1, &q->hrhs2, &q->frhs2, &q->vel1,
                     &q->vel2, &q->vel1p, &q->vel2p, &q->grad, &q->tmp[0], &q->tmp[1],
                     &q->tmp[2], &q->tmp[3]};
  se_advector* as[] = {q->adv1, q->adv2, q->adv1s, q->adv2s};
  for (se_advector* a : as)
    if (a) se_advector_destroy(a);
  se_linsys* ls[] = {q->helm1, q->helm2, q->fish1, q->fish2};
  for (se_linsys* l : ls)
    if (l) se_linsys_destroy(l);
  for (se_field** f : fs)
    if (*f) se_field_destroy(*f);
  delete q;
  return SE_OK;
}
#define QK(call)                  \
  do {                            \
    if (int rc_ = (call)) return rc_; \
  } while (0)

// One solve of a composed step; a solve that stops without converging leaves
// its last iterate in the field (as PETSc's KSPSolve does, whose callers in
// the reference never check) and is counted, and the step goes on.
int solve_counting(se_linsys* ls, int null, se_solve_stats* st, int* nc) {
  const int rc = se_linsys_solve(ls, null, st);
  if (rc == SE_ERR_NOT_CONVERGED) {
    ++*nc;
    return SE_OK;
  }
  return rc;
}

// PV advection of one layer into alpha_hat (first order: prev == nullptr).
int qg_advect(se_qg2* q, se_advector** adv, se_field* alpha, se_field* vel, se_field* alpha_p,
              se_field* vel_p, se_field* alpha_hat) {
  if (!*adv) QK(se_advector_create(alpha, vel, alpha_p, vel_p, adv));
  QK(se_advect(*adv, q->dt));
  return se_field_copy(alpha_hat, (*adv)->sl);
}

// Steps 2-4 (or 6-8) of the reference's step: baroclinic Helmholtz solve for
// t from a1 - a2, barotropic Poisson solve for c, then psi/omega from them.
int qg_invert(se_qg2* q, se_field* a1, se_field* a2, se_linsys* helm, se_field* hrhs, se_field* t,
              se_linsys* fish, se_field* frhs, se_field* c, double cb_fish, double cb_update,
              se_field* p1, se_field* p2, se_field* o1, se_field* o2) {
  const MeshDev& m = q->psi1->mesh->dev;
  CK(launch_qg_combine(m, 0, a1->vals, a2->vals, nullptr, nullptr, 0, 0, 0, hrhs->vals, nullptr,
                       nullptr, nullptr, g_stream));
  QK(solve_counting(helm, 0, nullptr, &q->nc));
  CK(launch_qg_combine(m, 1, a1->vals, a2->vals, t->vals, nullptr, q->F1, q->F2, cb_fish,
                       frhs->vals, nullptr, nullptr, nullptr, g_stream));
  QK(solve_counting(fish, 0, nullptr, &q->nc));
  CK(launch_qg_combine(m, 2, a1->vals, a2->vals, t->vals, c->vals, q->F1, q->F2, cb_update,
                       p1->vals, p2->vals, o1->vals, o2->vals, g_stream));
  return SE_OK;
}

int qg_status(const se_qg2* q) {
  if (q->nc) return fail(SE_ERR_NOT_CONVERGED, "%d of the step's solves did not converge", q->nc);
  return SE_OK;
}

// SolveQ of one layer: alpha (unknowns) = M^-1 DissipationRHS(alpha_hat, tau1, om_hat).
int qg_solve_q(se_qg2* q, se_field* alpha_hat, se_field* om_hat, double rF, double Ei,
               se_field* alpha) {
  const se_mesh* me = q->psi1->mesh;
  CK(launch_gen_vel(me->dev, om_hat->vals, q->grad->vals, nullptr, g_stream));
  CK(launch_qg_solve_q(me->dev, q->psi1->bcs->d[0], q->psi1->bcs->d[1], q->dt, alpha_hat->vals,
                       q->tau1->vals, om_hat->vals, q->grad->vals, q->tau_e->vals, rF, Ei, q->nu,
                       q->a_mass, alpha->vals, g_stream));
  return SE_OK;
}
}  // namespace

extern "C" {

int se_qg2_create(se_field* psi1, se_field* omega1, se_field* psi2, se_field* omega2, double F1,
                  double F2, double beta, double E2, double r, double nu, se_field* tau_e,
                  double dt, const se_solver_opts* opts, se_qg2** out) {
  if (!out) return fail(SE_ERR_ARG, "null argument");
  *out = nullptr;
  se_field* in[] = {psi1, omega1, psi2, omega2, tau_e};
  for (se_field* f : in) {
    if (int rc = check_field(f)) return rc;
    if (f->ndofs != 1 || f->mesh != psi1->mesh) return fail(SE_ERR_ARG, "fields must be scalar on one mesh");
  }
  if (!psi1->bcs) return fail(SE_ERR_ARG, "psi1 needs boundary conditions");
  if (psi1->mesh->dev.N < 3) return fail(SE_ERR_UNSUPPORTED, "N < 3 SL is not built");
  se_qg2* q = new se_qg2();
  std::memset((void*)q, 0, sizeof(*q));
  q->psi1 = psi1;
  q->omega1 = omega1;
  q->psi2 = psi2;
  q->omega2 = omega2;
  q->tau_e = tau_e;
  q->F1 = F1;
  q->F2 = F2;
  q->beta = beta;
  q->E2 = E2;
  q->r = r;
  q->nu = nu;
  q->dt = dt;
  q->a_mass = 1.0;
  se_mesh* me = psi1->mesh;
  se_bcs* bc = psi1->bcs;
  se_field** with_bc[] = {&q->tau1, &q->chi1, &q->tau2, &q->chi2, &q->psi1h, &q->psi2h, &q->om1h,
                          &q->om2h, &q->alpha1, &q->alpha2, &q->alpha1h, &q->alpha2h};
  se_field** no_bc[] = {&q->alpha1p, &q->alpha2p, &q->hrhs1, &q->frhs1, &q->hrhs2, &q->frhs2,
                        &q->tmp[0], &q->tmp[1], &q->tmp[2], &q->tmp[3]};
  se_field** two[] = {&q->vel1, &q->vel2, &q->vel1p, &q->vel2p, &q->grad};
  int rc = SE_OK;
  for (se_field** f : with_bc)
    if (!rc) rc = se_field_create(me, 1, bc, f);
  for (se_field** f : no_bc)
    if (!rc) rc = se_field_create(me, 1, nullptr, f);
  for (se_field** f : two)
    if (!rc) rc = se_field_create(me, 2, nullptr, f);
  // boundary values of the baroclinic (tau = psi1 - psi2) and barotropic
  // (chi = psi1 + psi2) stream functions (src/qg/TwoLayerQGEqn.cpp:46-53)
  const MeshDev& m = me->dev;
  if (!rc && (launch_qg_combine(m, 0, psi1->vals, psi2->vals, nullptr, nullptr, 0, 0, 0,
                                q->tau1->vals, nullptr, nullptr, nullptr, g_stream) ||
              launch_qg_combine(m, 0, psi1->vals, psi2->vals, nullptr, nullptr, 0, 0, 0,
                                q->tau2->vals, nullptr, nullptr, nullptr, g_stream)))
    rc = fail(SE_ERR_CUDA, "QG set-up launch failed");
  // chi = psi1 + psi2: the Poisson combination with zero coefficients
  if (!rc && (launch_qg_combine(m, 1, psi1->vals, psi2->vals, psi1->vals, nullptr, 0, 0, 0,
                                q->chi1->vals, nullptr, nullptr, nullptr, g_stream) ||
              launch_qg_combine(m, 1, psi1->vals, psi2->vals, psi1->vals, nullptr, 0, 0, 0,
                                q->chi2->vals, nullptr, nullptr, nullptr, g_stream)))
    rc = fail(SE_ERR_CUDA, "QG set-up launch failed");
  const double cmass = -(F1 + F2);
  if (!rc) rc = se_helmholtz_create(q->tau1, q->hrhs1, cmass, -1.0, 1.0, 0, opts, &q->helm1);
  if (!rc) rc = se_helmholtz_create(q->tau2, q->hrhs2, cmass, -1.0, 1.0, 0, opts, &q->helm2);
  if (!rc) rc = se_poisson_create(q->chi1, q->frhs1, -1.0, opts, &q->fish1);
  if (!rc) rc = se_poisson_create(q->chi2, q->frhs2, -1.0, opts, &q->fish2);
  // the PV fields (src/qg/TwoLayerQGEqn.cpp:71-72)
  if (!rc && (launch_gen_pv(m, omega1->vals, psi1->vals, psi2->vals, F1, beta, q->alpha1->vals,
                            g_stream) ||
              launch_gen_pv(m, omega2->vals, psi2->vals, psi1->vals, F2, beta, q->alpha2->vals,
                            g_stream)))
    rc = fail(SE_ERR_CUDA, "QG set-up launch failed");
  if (rc) {
    qg_release(q);
    return rc;
  }
  *out = q;
  return SE_OK;
}

int se_qg2_destroy(se_qg2* q) {
  if (!q) return SE_OK;
  return qg_release(q);
}

int se_qg2_solve(se_qg2* q, se_field* psi1p, se_field* omega1p, se_field* psi2p,
                 se_field* omega2p) {
  if (!q) return fail(SE_ERR_ARG, "null QG system");
  const MeshDev& m = q->psi1->mesh->dev;
  const bool second = psi1p && omega1p && psi2p && omega2p;
  q->nc = 0;
  if (second) {
    se_field* pv[] = {psi1p, omega1p, psi2p, omega2p};
    for (se_field* f : pv) {
      if (int rc = check_field(f)) return rc;
      if (f->ndofs != 1 || f->mesh != q->psi1->mesh) return fail(SE_ERR_ARG, "previous fields do not match");
    }
  }
  if (!second) {
    // TwoLayerQGEqn::FirstOrder (src/qg/TwoLayerQGEqn.cpp:175-243)
    CK(launch_gen_vel(m, q->psi1->vals, q->vel1->vals, nullptr, g_stream));
    CK(launch_gen_vel(m, q->psi2->vals, q->vel2->vals, nullptr, g_stream));
    CK(launch_gen_pv(m, q->omega1->vals, q->psi1->vals, q->psi2->vals, q->F1, q->beta,
                     q->alpha1->vals, g_stream));
    CK(launch_gen_pv(m, q->omega2->vals, q->psi2->vals, q->psi1->vals, q->F2, q->beta,
                     q->alpha2->vals, g_stream));
    QK(qg_advect(q, &q->adv1, q->alpha1, q->vel1, nullptr, nullptr, q->alpha1h));
    QK(qg_advect(q, &q->adv2, q->alpha2, q->vel2, nullptr, nullptr, q->alpha2h));
    QK(qg_invert(q, q->alpha1h, q->alpha2h, q->helm1, q->hrhs1, q->tau1, q->fish1, q->frhs1,
                 q->chi1, 2.0 * q->beta, q->beta, q->psi1h, q->psi2h, q->om1h, q->om2h));
    QK(qg_solve_q(q, q->alpha1h, q->om1h, q->r * q->F1, 0.0, q->alpha1));
    QK(qg_invert(q, q->alpha1, q->alpha2, q->helm2, q->hrhs2, q->tau2, q->fish2, q->frhs2,
                 q->chi2, 2.0 * q->beta, q->beta, q->psi1, q->psi2, q->omega1, q->omega2));
    return qg_status(q);
  }
  // TwoLayerQGEqn::Solve with previous fields (src/qg/TwoLayerQGEqn.cpp:123-172)
  if (!q->second_assembled) {
    q->a_mass = 1.5;
    q->second_assembled = true;
  }
  QK(se_field_copy(q->tmp[0], q->psi1));
  QK(se_field_copy(q->tmp[1], q->psi2));
  QK(se_field_copy(q->tmp[2], q->omega1));
  QK(se_field_copy(q->tmp[3], q->omega2));
  // TwoLayerQGEqn::SecondOrder (src/qg/TwoLayerQGEqn.cpp:245-324)
  const double a = 1.5;
  CK(launch_gen_vel(m, q->psi1->vals, q->vel1->vals, nullptr, g_stream));
  CK(launch_gen_vel(m, q->psi2->vals, q->vel2->vals, nullptr, g_stream));
  CK(launch_gen_vel(m, psi1p->vals, q->vel1p->vals, nullptr, g_stream));
  CK(launch_gen_vel(m, psi2p->vals, q->vel2p->vals, nullptr, g_stream));
  CK(launch_gen_pv(m, q->omega1->vals, q->psi1->vals, q->psi2->vals, q->F1, q->beta,
                   q->alpha1->vals, g_stream));
  CK(launch_gen_pv(m, q->omega2->vals, q->psi2->vals, q->psi1->vals, q->F2, q->beta,
                   q->alpha2->vals, g_stream));
  CK(launch_gen_pv(m, omega1p->vals, psi1p->vals, psi2p->vals, q->F1, q->beta, q->alpha1p->vals,
                   g_stream));
  CK(launch_gen_pv(m, omega2p->vals, psi2p->vals, psi1p->vals, q->F2, q->beta, q->alpha2p->vals,
                   g_stream));
  QK(qg_advect(q, &q->adv1s, q->alpha1, q->vel1, q->alpha1p, q->vel1p, q->alpha1h));
  QK(qg_advect(q, &q->adv2s, q->alpha2, q->vel2, q->alpha2p, q->vel2p, q->alpha2h));
  QK(qg_invert(q, q->alpha1h, q->alpha2h, q->helm1, q->hrhs1, q->tau1, q->fish1, q->frhs1,
               q->chi1, a * 2.0 * q->beta, a * q->beta, q->psi1h, q->psi2h, q->om1h, q->om2h));
  QK(qg_solve_q(q, q->alpha1h, q->om1h, q->r * q->F1, 0.0, q->alpha1));
  QK(qg_solve_q(q, q->alpha2h, q->om2h, -q->r * q->F2, q->E2, q->alpha2));
  QK(qg_invert(q, q->alpha1, q->alpha2, q->helm2, q->hrhs2, q->tau2, q->fish2, q->frhs2, q->chi2,
               2.0 * q->beta, q->beta, q->psi1, q->psi2, q->omega1, q->omega2));
  QK(se_field_copy(psi1p, q->tmp[0]));
  QK(se_field_copy(psi2p, q->tmp[1]));
  QK(se_field_copy(omega1p, q->tmp[2]));
  QK(se_field_copy(omega2p, q->tmp[3]));
  return qg_status(q);
}

}  // extern "C"

// ------------------------------------------- Navier-Stokes splitting step --
// NavierStokesEqn (src/ns/NavierStokesEqn.cpp:23-147) composed from this
// library's objects: the SL advector (velocity by itself), the divergence and
// pressure-gradient kernels (sl.cu), the pressure PoissonEqn(pressure,
// divVelStep1, -dt) solved with the constant null space removed, and the
// viscous HelmholtzEqn(velocity, velStep2, c, nu, dt) as one scalar system
// per velocity component (the reference's interleaved system is block
// diagonal per component). As in the reference, the viscous systems are made
// (and their Dirichlet values taken from the velocity) on the first
// first-order step with c = 1.0 and again on the first second-order step with
// c = 1.5; the pressure system is made once.
struct se_ns {
  se_field *velocity, *pressure;  // the caller's
  se_bcs *bcs_u, *bcs_v;          // the caller's (may be null)
  double dt;
  se_solver_opts opts;
  bool second_done;
  se_field *div, *step2;     // divVelStep1 (1 component), velStep2 (2 components)
  se_field *u, *v, *ru, *rv; // velocity components and their right-hand sides
  se_linsys *poisson, *hu, *hv;
  se_advector *adv1, *adv2;  // first order; second order (previous velocity set per call)
  unsigned* err;
  se_solve_stats st[3];
};

namespace {
bool same_geometry(const se_mesh* a, const se_mesh* b) {
  if (a == b) return true;
  const MeshDev &x = a->dev, &y = b->dev;
  return x.N == y.N && x.nEls[0] == y.nEls[0] && x.nEls[1] == y.nEls[1] &&
         x.periodic[0] == y.periodic[0] && x.periodic[1] == y.periodic[1] &&
         x.min[0] == y.min[0] && x.min[1] == y.min[1] && x.max[0] == y.max[0] &&
         x.max[1] == y.max[1];
}

int ns_release(se_ns* n) {
  se_advector* as[] = {n->adv1, n->adv2};
  for (se_advector* a : as)
    if (a) se_advector_destroy(a);
  se_linsys* ls[] = {n->poisson, n->hu, n->hv};
  for (se_linsys* l : ls)
    if (l) se_linsys_destroy(l);
  se_field* fs[] = {n->div, n->step2, n->u, n->v, n->ru, n->rv};
  for (se_field* f : fs)
    if (f) se_field_destroy(f);
  dfree(n->err);
  delete n;
  return SE_OK;
}

// (Re)make the two viscous systems with mass coefficient c (and the SVV
// operator when svv != 0, which only CG solves: the fast diagonalization does
// not hold for it, so those two systems use CG whatever the options' method).
int ns_make_viscous(se_ns* n, double c, double nu, int svv) {
  if (n->hu) se_linsys_destroy(n->hu);
  if (n->hv) se_linsys_destroy(n->hv);
  n->hu = n->hv = nullptr;
  se_solver_opts o = n->opts;
  if (svv) o.method = SE_METHOD_CG, o.precision = SE_PREC_FP64;
  QK(se_helmholtz_create(n->u, n->ru, c, nu, n->dt, svv, &o, &n->hu));
  return se_helmholtz_create(n->v, n->rv, c, nu, n->dt, svv, &o, &n->hv);
}
}  // namespace

extern "C" {

int se_ns_create(se_field* velocity, se_field* pressure, se_bcs* bcs_u, se_bcs* bcs_v, double dt,
                 const se_solver_opts* opts, se_ns** out) {
  if (!out) return fail(SE_ERR_ARG, "null argument");
  *out = nullptr;
  if (int rc = check_field(velocity)) return rc;
  if (int rc = check_field(pressure)) return rc;
  if (velocity->ndofs != 2 || pressure->ndofs != 1)
    return fail(SE_ERR_ARG, "velocity needs 2 components and pressure 1");
  if (!same_geometry(velocity->mesh, pressure->mesh))
    return fail(SE_ERR_UNSUPPORTED, "pressure mesh of another geometry is not built");
  se_bcs* bs[] = {bcs_u, bcs_v};
  for (se_bcs* b : bs)
    if (b && b->mesh != velocity->mesh) return fail(SE_ERR_ARG, "component BCs on another mesh");
  if (velocity->mesh->dev.N < 3) return fail(SE_ERR_UNSUPPORTED, "N < 3 SL is not built");
  se_solver_opts o;
  if (opts) {
    if (int rc = check_opts(opts)) return rc;
    o = *opts;
  } else {
    se_solver_opts_default(&o);
  }
  se_ns* n = new se_ns();
  std::memset((void*)n, 0, sizeof(*n));
  n->velocity = velocity;
  n->pressure = pressure;
  n->bcs_u = bcs_u;
  n->bcs_v = bcs_v;
  n->dt = dt;
  n->opts = o;
  se_mesh* me = velocity->mesh;
  int rc = dalloc(&n->err, 1);
  if (!rc) rc = se_field_create(pressure->mesh, 1, nullptr, &n->div);
  if (!rc) rc = se_field_create(me, 2, nullptr, &n->step2);
  if (!rc) rc = se_field_create(me, 1, bcs_u, &n->u);
  if (!rc) rc = se_field_create(me, 1, bcs_v, &n->v);
  if (!rc) rc = se_field_create(me, 1, nullptr, &n->ru);
  if (!rc) rc = se_field_create(me, 1, nullptr, &n->rv);
  if (!rc) rc = se_poisson_create(pressure, n->div, -dt, &n->opts, &n->poisson);
  if (rc) {
    ns_release(n);
    return rc;
  }
  *out = n;
  return SE_OK;
}

int se_ns_solve(se_ns* n, se_field* velocity, se_field* pressure, se_field* prev_vel, double nu,
                int svvCutoff) {
  if (!n) return fail(SE_ERR_ARG, "null Navier-Stokes system");
  if (velocity != n->velocity || pressure != n->pressure)
    return fail(SE_ERR_ARG, "velocity and pressure must be the fields the system was made with");
  if (svvCutoff < 0 || svvCutoff > velocity->mesh->dev.N)
    return fail(SE_ERR_ARG, "svvCutoff %d outside [0, N]", svvCutoff);
  const bool second = prev_vel != nullptr;
  if (second) {
    if (int rc = check_field(prev_vel)) return rc;
    if (prev_vel->ndofs != 2 || prev_vel->mesh != velocity->mesh)
      return fail(SE_ERR_ARG, "previous velocity does not match");
  }
  const se_mesh* me = velocity->mesh;
  const MeshDev& m = me->dev;
  const int nv = me->nVertsTotal;
  // advective step: the velocity advected by itself (a new Advector per step
  // in the reference; here one per order, the previous velocity set per call)
  se_advector** adv = second ? &n->adv2 : &n->adv1;
  if (!*adv) QK(se_advector_create(velocity, velocity, prev_vel, prev_vel, adv));
  (*adv)->field_prev = prev_vel;
  (*adv)->vel_prev = prev_vel;
  QK(se_advect(*adv, n->dt));
  const double* sl = (*adv)->sl->vals;
  // pressure step
  CK(cudaMemsetAsync(n->err, 0, sizeof(unsigned), g_stream));
  CK(launch_ns_pressure(m, second ? 2 : 0, sl, nullptr, 0.0, n->div->vals, n->err, g_stream));
  int nc = 0;  // solves that stopped without converging (the step goes on, as in the reference)
  QK(solve_counting(n->poisson, 2, &n->st[0], &nc));
  CK(launch_ns_pressure(m, 1, sl, pressure->vals, n->dt, n->step2->vals, n->err, g_stream));
  // viscous step
  if (!second && !n->hu) QK(ns_make_viscous(n, 1.0, nu, svvCutoff));
  if (second && !n->second_done) QK(ns_make_viscous(n, 1.5, nu, svvCutoff));
  CK(launch_component(nv, 1, 0, velocity->vals, n->u->vals, g_stream));
  CK(launch_component(nv, 1, 1, velocity->vals, n->v->vals, g_stream));
  CK(launch_component(nv, 1, 0, n->step2->vals, n->ru->vals, g_stream));
  CK(launch_component(nv, 1, 1, n->step2->vals, n->rv->vals, g_stream));
  QK(solve_counting(n->hu, 0, &n->st[1], &nc));
  QK(solve_counting(n->hv, 0, &n->st[2], &nc));
  CK(launch_component(nv, 0, 0, velocity->vals, n->u->vals, g_stream));
  CK(launch_component(nv, 0, 1, velocity->vals, n->v->vals, g_stream));
  if (second) n->second_done = true;
  unsigned herr = 0;
  CK(cudaMemcpyAsync(&herr, n->err, sizeof(unsigned), cudaMemcpyDeviceToHost, g_stream));
  CK(cudaStreamSynchronize(g_stream));
  if (herr) return fail(SE_ERR_CUDA, "Navier-Stokes derivative kernel error bits 0x%x", herr);
  if (nc)
    return fail(SE_ERR_NOT_CONVERGED, "%d of the step's solves did not converge (reasons %d %d %d)",
                nc, n->st[0].reason, n->st[1].reason, n->st[2].reason);
  return SE_OK;
}

int se_ns_stats(const se_ns* n, se_solve_stats stats[3]) {
  if (!n || !stats) return fail(SE_ERR_ARG, "null argument");
  for (int k = 0; k < 3; k++) stats[k] = n->st[k];
  return SE_OK;
}

int se_ns_destroy(se_ns* n) {
  if (!n) return SE_OK;
  return ns_release(n);
}

}  // extern "C"
#undef QK
