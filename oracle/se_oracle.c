/* CPU restatement of SE's semi-Lagrangian + Helmholtz/Poisson hot path.
 *
 * TEST INFRASTRUCTURE ONLY (the oracle and the timed CPU baseline); the
 * product never links or calls this file. Every function cites the
 * reference code it restates (paths relative to the SE checkout). Where the
 * reference's floating-point operation order matters for bit parity, the
 * restatement keeps it, and it is compiled without FMA contraction like the
 * reference, so that the two agree bit for bit (tests/test_oracle_pin.py).
 */
#define _GNU_SOURCE
#include "se_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#define MAXN 17 /* largest polynomial order handled */

/* Static-chunk parallel loop over [0, n) on nthreads POSIX threads. Each
 * chunk is a contiguous range, so per-index work is independent of the
 * thread count. */
typedef void (*range_fn)(void* ctx, long b, long e, int t);
typedef struct { range_fn fn; void* ctx; long b, e; int t; } range_job;
static void* range_run(void* p) {
  range_job* j = (range_job*)p;
  j->fn(j->ctx, j->b, j->e, j->t);
  return NULL;
}
static void par_for(int nthreads, long n, range_fn fn, void* ctx) {
  int nt = nthreads > 0 ? nthreads : 1;
  if (nt > 256) nt = 256;
  if (nt == 1 || n < 2) {
    fn(ctx, 0, n, 0);
    return;
  }
  pthread_t th[256];
  range_job jobs[256];
  for (int t = 0; t < nt; t++) {
    jobs[t].fn = fn;
    jobs[t].ctx = ctx;
    jobs[t].b = n * t / nt;
    jobs[t].e = n * (t + 1) / nt;
    jobs[t].t = t;
    if (t > 0) pthread_create(&th[t], NULL, range_run, &jobs[t]);
  }
  range_run(&jobs[0]);
  for (int t = 1; t < nt; t++) pthread_join(th[t], NULL);
}

struct or_mesh {
  int N, n, nn;
  int nEls[2], nVerts[2], nVertsTotal, nElsTotal;
  int periodic[2];
  double min[2], max[2], dx[2];
  double abcissa[MAXN + 1], weights[MAXN + 1];
  double dC[(MAXN + 1) * (MAXN + 1)];
  double Pc[MAXN + 2]; /* monomial coefficients of P_N */
  double* verts;       /* [nVertsTotal][2] */
  int accurate;        /* 1: cardinal functions in extended precision */
};

/* ---------------------------------------------------------------- Jacobi --
 * src/base/Jacobi.cpp:34-89: Legendre polynomials as monomial coefficient
 * arrays built by the three-term recurrence, evaluated with pow() summing only
 * the terms of matching parity. */
static void jac_gen(int n, double a, const double* m1, int n1, const double* m2,
                    int n2, double* c) {
  int i;
  double c1 = 2 * n * (2 * a + n) * (2 * a + 2 * n - 2);
  double c2 = (2 * a + 2 * n - 1) * (2 * a + 2 * n) * (2 * a + 2 * n - 2);
  double c3 = 2 * (a + n - 1) * (a + n - 1) * (2 * a + 2 * n);
  c2 /= c1;
  c3 /= c1;
  for (i = 0; i <= n1; i++) c[i + 1] += c2 * m1[i];
  for (i = 0; i <= n2; i++) c[i] -= c3 * m2[i];
}
static double jac_eval(int n, const double* c, double x) {
  double p = 0.0;
  for (int i = n; i >= 0; i -= 2) p += c[i] * pow(x, i);
  return p;
}
static double jac_deriv(int n, const double* c, double x) {
  double dp = 0.0;
  for (int i = n; i >= 1; i -= 2) dp += c[i] * i * pow(x, i - 1);
  return dp;
}
static double jac_deriv2(int n, const double* c, double x) {
  double d2p = 0.0;
  for (int i = n; i >= 2; i -= 2) d2p += c[i] * i * (i - 1) * pow(x, i - 2);
  return d2p;
}

/* src/base/Element.cpp:54-64 (Newton on P_N', tolerance 1e-12). The
 * reference loops until converged; the cap only guards this port. */
static double root_finder(double x0, int N, const double* c) {
  double x = x0, xp;
  for (int it = 0; it < 100000; it++) {
    xp = x;
    x = xp - jac_deriv(N, c, xp) / jac_deriv2(N, c, xp);
    if (fabs(x - xp) < 1.0e-12) return x;
  }
  return x;
}
/* src/base/Element.cpp:66-75 */
static int already_found(int n, const double* roots, double root) {
  for (int i = 0; i < n; i++)
    if (fabs(roots[i] - root) < 1.0e-6) return 1;
  return 0;
}
/* src/base/Element.cpp:77-106 (selection sort, ascending) */
static void sort_entries(double* vals, int n) {
  int done[MAXN + 1] = {0};
  double temp[MAXN + 1];
  int minInd = 0;
  for (int i = 0; i < n; i++) {
    double minVal = 1.0e+99;
    for (int j = 0; j < n; j++)
      if (!done[j] && vals[j] < minVal) {
        minVal = vals[j];
        minInd = j;
      }
    temp[i] = minVal;
    done[minInd] = 1;
  }
  for (int i = 0; i < n; i++) vals[i] = temp[i];
}

/* src/base/Legendre.cpp:15-95: GLL nodes (roots of P_N' by Newton from the
 * left, mirrored), weights 2/(N(N+1)P_N(x)^2) and the cardinal-derivative
 * matrix dCij (row = point, column = basis). Fills the mesh's tables. */
static void legendre_tables(int N, double* abcissa, double* weights, double* dC,
                            double* Pc) {
  double polys[MAXN + 3][MAXN + 3];
  memset(polys, 0, sizeof(polys));
  polys[0][0] = 1.0;
  polys[1][1] = 1.0;
  for (int i = 2; i <= N + 1; i++) jac_gen(i, 0.0, polys[i - 1], i - 1, polys[i - 2], i - 2, polys[i]);
  const double* PN = polys[N];
  double STEP = 1.0e-3;
  abcissa[0] = -1.0;
  int endLoop = ((N + 1) % 2 == 1) ? N / 2 : (N + 1) / 2;
  for (int i = 1; i < endLoop; i++) {
    double x0 = abcissa[i - 1];
    do {
      x0 += STEP;
      abcissa[i] = root_finder(x0, N, PN);
    } while (already_found(i, abcissa, abcissa[i]) || abcissa[i] > 0.0 - STEP);
    abcissa[N - i] = -abcissa[i];
  }
  abcissa[N] = 1.0;
  if ((N + 1) % 2 == 1) abcissa[(N + 1) / 2] = 0.0;
  sort_entries(abcissa, N + 1);
  weights[0] = 2.0 / ((N + 1) * N);
  for (int i = 1; i < N; i++)
    weights[i] = 2.0 / ((N + 1) * N * jac_eval(N, PN, abcissa[i]) * jac_eval(N, PN, abcissa[i]));
  weights[N] = 2.0 / ((N + 1) * N);
  /* P = Jacobi(N).Gen(polys[N-1], polys[N-2]) has the coefficients of polys[N] */
  double P[MAXN + 2];
  memset(P, 0, sizeof(P));
  jac_gen(N, 0.0, polys[N - 1], N - 1, polys[N - 2], N - 2, P);
  memcpy(Pc, P, sizeof(double) * (N + 1));
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
        v = jac_eval(N, P, abcissa[i]) / (jac_eval(N, P, abcissa[j]) * (abcissa[i] - abcissa[j]));
      dC[i * (N + 1) + j] = v;
    }
}

void or_gll(int N, double* abcissa, double* weights, double* dCij, double* Pj) {
  double Pc[MAXN + 2];
  legendre_tables(N, abcissa, weights, dCij, Pc);
  for (int i = 0; i <= N; i++) Pj[i] = jac_eval(N, Pc, abcissa[i]);
}

/* ------------------------------------------------------------------ Mesh --
 * src/base/Mesh.cpp:17-84: regular nEls[0] x nEls[1] mesh of order-N
 * elements, (nEls*N+1)^2 vertices, periodic duplicates stored. */
or_mesh* or_mesh_create(int nx, int ny, int N, double x0, double y0, double x1,
                        double y1, int perx, int pery) {
  if (N < 2 || N > MAXN || nx < 1 || ny < 1) return NULL;
  or_mesh* m = (or_mesh*)calloc(1, sizeof(or_mesh));
  m->N = N;
  m->n = N + 1;
  m->nn = (N + 1) * (N + 1);
  legendre_tables(N, m->abcissa, m->weights, m->dC, m->Pc);
  int ne[2] = {nx, ny};
  double mn[2] = {x0, y0}, mx[2] = {x1, y1};
  int per[2] = {perx != 0, pery != 0};
  for (int d = 0; d < 2; d++) {
    m->nEls[d] = ne[d];
    m->nVerts[d] = ne[d] * N + 1;
    m->min[d] = mn[d];
    m->max[d] = mx[d];
    m->periodic[d] = per[d];
    m->dx[d] = (m->max[d] - m->min[d]) / m->nEls[d];
  }
  m->nElsTotal = m->nEls[0] * m->nEls[1];
  m->nVertsTotal = m->nVerts[0] * m->nVerts[1];
  m->verts = (double*)malloc(sizeof(double) * 2 * m->nVertsTotal);
  for (int v = 0; v < m->nVertsTotal; v++) {
    int t0 = v % m->nVerts[0], t1 = v / m->nVerts[0];
    int ei = t0 / N, ej = t1 / N;
    double l0 = m->abcissa[t0 % N], l1 = m->abcissa[t1 % N];
    m->verts[2 * v] = m->min[0] + ei * m->dx[0] + ((l0 + 1.0) / 2.0) * m->dx[0];
    m->verts[2 * v + 1] = m->min[1] + ej * m->dx[1] + ((l1 + 1.0) / 2.0) * m->dx[1];
  }
  return m;
}
void or_mesh_destroy(or_mesh* m) {
  if (!m) return;
  free(m->verts);
  free(m);
}
int or_mesh_nverts(const or_mesh* m) { return m->nVertsTotal; }
void or_mesh_verts(const or_mesh* m, double* out) {
  memcpy(out, m->verts, sizeof(double) * 2 * m->nVertsTotal);
}

/* src/base/Mesh.cpp:138-152 */
static void el_nodes(const or_mesh* m, int el, int* nodes) {
  int N = m->N, t0 = N * (el % m->nEls[0]), t1 = N * (el / m->nEls[0]);
  int n0 = t1 * m->nVerts[0] + t0, k = 0;
  for (int jj = 0; jj < N + 1; jj++)
    for (int ii = 0; ii < N + 1; ii++) nodes[k++] = n0 + jj * m->nVerts[0] + ii;
}

#define EPSILON 1.0e-12
#define NUMAPPROX(var, val) ((var) >= (val)-EPSILON && (var) <= (val) + EPSILON)

/* src/base/Mesh.cpp:109-136: element search with the 1e-12 snap onto the
 * lower element at interior element edges and onto the last element at max. */
static int get_el(const or_mesh* m, const double* c) {
  int topo[2];
  for (int d = 0; d < 2; d++) {
    if (NUMAPPROX(c[d] - m->max[d], 0.0)) {
      topo[d] = m->nEls[d] - 1;
    } else {
      double out = (c[d] - m->min[d]) / m->dx[d], integer;
      double frac = modf(out, &integer);
      topo[d] = (int)integer;
      if (topo[d] > 0 && NUMAPPROX(frac, 0.0)) topo[d]--;
    }
  }
  return topo[1] * m->nEls[0] + topo[0];
}
/* src/base/Mesh.cpp:163-176 */
static int global_to_local(const or_mesh* m, const double* g, double* l) {
  int el = get_el(m, g);
  l[0] = (g[0] - m->min[0] - (el % m->nEls[0]) * m->dx[0]) * (2.0 / m->dx[0]) - 1.0;
  l[1] = (g[1] - m->min[1] - (el / m->nEls[0]) * m->dx[1]) * (2.0 / m->dx[1]) - 1.0;
  for (int d = 0; d < 2; d++) {
    if (l[d] < -1.0) l[d] = -1;
    if (l[d] > +1.0) l[d] = +1;
  }
  return el;
}
void or_global_to_local(const or_mesh* m, const double* pts, int npts, int* el,
                        double* lc) {
  for (int k = 0; k < npts; k++) el[k] = global_to_local(m, pts + 2 * k, lc + 2 * k);
}

/* src/base/Legendre.cpp:293-305: a coordinate within 1e-8 of a GLL node is
 * that node. */
static int is_root(const or_mesh* m, double x, int* i) {
  for (int k = 0; k <= m->N; k++)
    if (fabs(x - m->abcissa[k]) < 1.0e-8) {
      *i = k;
      return 1;
    }
  *i = -1;
  return 0;
}

/* src/base/Legendre.cpp:145-169: GLL cardinal functions at a local point,
 * node index x fastest. */
static void shape_funcs_at(const or_mesh* m, const double* c, double* Ni) {
  int N = m->N, xi, yi;
  for (int pt = 0; pt < m->nn; pt++) {
    int xj = pt % (N + 1), yj = pt / (N + 1);
    double Nx, Ny;
    if (is_root(m, c[0], &xi))
      Nx = (xi == xj) ? 1.0 : 0.0;
    else
      Nx = -((1.0 - c[0] * c[0]) /
             (N * (N + 1) * jac_eval(N, m->Pc, m->abcissa[xj]) * (c[0] - m->abcissa[xj]))) *
           jac_deriv(N, m->Pc, c[0]);
    if (is_root(m, c[1], &yi))
      Ny = (yi == yj) ? 1.0 : 0.0;
    else
      Ny = -((1.0 - c[1] * c[1]) /
             (N * (N + 1) * jac_eval(N, m->Pc, m->abcissa[yj]) * (c[1] - m->abcissa[yj]))) *
           jac_deriv(N, m->Pc, c[1]);
    Ni[pt] = Nx * Ny;
  }
}
void or_shape_funcs_at(const or_mesh* m, const double* coords, int npts, double* Ni) {
  for (int k = 0; k < npts; k++) shape_funcs_at(m, coords + 2 * k, Ni + (size_t)k * m->nn);
}

/* Extended-precision variant of the interpolation, a test switch that is
 * not part of the reference: the same element search, local coordinates and
 * 1e-8 node snap, but the cardinal functions as Lagrange products and the
 * sum in long double. The reference's own formula evaluates P_N'(x) as a
 * monomial sum, which cancels near the GLL nodes (relative error up to
 * ~1e-16 * C / |x - x_k|, i.e. ~1e-8 at the snap radius); this variant is
 * accurate to rounding and measures how close a faster evaluation is to
 * the reference's mathematics. */
static void interp_accurate(const or_mesh* m, int ndofs, const double* vals, int el,
                            const double* l, double* val) {
  int N = m->N, snap[2];
  long double c[2][MAXN + 1];
  for (int d = 0; d < 2; d++) {
    if (is_root(m, l[d], &snap[d])) {
      for (int j = 0; j <= N; j++) c[d][j] = (j == snap[d]) ? 1.0L : 0.0L;
    } else {
      for (int j = 0; j <= N; j++) {
        long double p = 1.0L;
        for (int k = 0; k <= N; k++)
          if (k != j)
            p *= ((long double)l[d] - (long double)m->abcissa[k]) /
                 ((long double)m->abcissa[j] - (long double)m->abcissa[k]);
        c[d][j] = p;
      }
    }
  }
  int nodes[(MAXN + 1) * (MAXN + 1)];
  el_nodes(m, el, nodes);
  for (int d = 0; d < ndofs; d++) {
    long double s = 0.0L;
    for (int k = 0; k < m->nn; k++)
      s += c[0][k % (N + 1)] * c[1][k / (N + 1)] * (long double)vals[(size_t)nodes[k] * ndofs + d];
    val[d] = (double)s;
  }
}

void or_mesh_set_accurate(or_mesh* m, int on) { m->accurate = on != 0; }

/* src/base/Field.cpp:57-76 */
static void interp_global(const or_mesh* m, int ndofs, const double* vals,
                          const double* g, double* val) {
  double l[2], Ni[(MAXN + 1) * (MAXN + 1)];
  int nodes[(MAXN + 1) * (MAXN + 1)];
  int el = global_to_local(m, g, l);
  if (m->accurate) {
    interp_accurate(m, ndofs, vals, el, l, val);
    return;
  }
  shape_funcs_at(m, l, Ni);
  el_nodes(m, el, nodes);
  for (int d = 0; d < ndofs; d++) val[d] = 0.0;
  for (int k = 0; k < m->nn; k++)
    for (int d = 0; d < ndofs; d++) val[d] += Ni[k] * vals[(size_t)nodes[k] * ndofs + d];
}
void or_interp_global(const or_mesh* m, int ndofs, const double* vals,
                      const double* pts, int npts, double* out) {
  for (int k = 0; k < npts; k++) interp_global(m, ndofs, vals, pts + 2 * k, out + (size_t)k * ndofs);
}

/* ------------------------------------------------------------- Advector -- */
/* src/base/Advector.cpp:122-134: one periodic wrap, or a clamp at walls. */
static void sl_periodic_update(const or_mesh* m, double* c) {
  for (int d = 0; d < 2; d++) {
    if (c[d] < m->min[d]) c[d] = m->periodic[d] ? m->max[d] - m->min[d] + c[d] : m->min[d];
    if (c[d] > m->max[d]) c[d] = m->periodic[d] ? m->min[d] - m->max[d] + c[d] : m->max[d];
  }
}
/* src/base/Advector.cpp:136-148: midpoint RK2 backward trajectory; the first
 * stage always uses the current velocity. */
static void integrate_rk2(const or_mesh* m, double dt, const double* vel,
                          const double* velField, const double* origin, double* coord) {
  double xHat[2], v[2];
  interp_global(m, 2, vel, origin, v);
  xHat[0] = origin[0] - 0.5 * dt * v[0];
  xHat[1] = origin[1] - 0.5 * dt * v[1];
  sl_periodic_update(m, xHat);
  interp_global(m, 2, velField, xHat, v);
  coord[0] = origin[0] - dt * v[0];
  coord[1] = origin[1] - dt * v[1];
  sl_periodic_update(m, coord);
}
/* src/base/Field.cpp:232-252 */
void or_periodic_update(const or_mesh* m, int ndofs, double* vals) {
  int nx = m->nVerts[0], ny = m->nVerts[1];
  if (m->periodic[0])
    for (int j = 0; j < ny; j++)
      for (int d = 0; d < ndofs; d++)
        vals[(size_t)(j * nx + nx - 1) * ndofs + d] = vals[(size_t)(j * nx) * ndofs + d];
  if (m->periodic[1])
    for (int i = 0; i < nx; i++)
      for (int d = 0; d < ndofs; d++)
        vals[(size_t)(nx * (ny - 1) + i) * ndofs + d] = vals[(size_t)i * ndofs + d];
  if (m->periodic[0] && m->periodic[1])
    for (int d = 0; d < ndofs; d++) vals[(size_t)(nx * ny - 1) * ndofs + d] = vals[d];
}

/* src/base/Advector.cpp:339-349 */
static void extrapolate(int nv, const double* v, const double* vm, double* p1,
                        double* ph, double* mh) {
  for (int k = 0; k < 2 * nv; k++) {
    p1[k] = 2.0 * v[k] - 1.0 * vm[k];
    ph[k] = 1.5 * v[k] - 0.5 * vm[k];
    mh[k] = 0.5 * v[k] + 0.5 * vm[k];
  }
}
/* src/base/Advector.cpp:203-228: second-order two-step trajectory. */
static void trajectory2(const or_mesh* m, double dt, const double* vel,
                        const double* p1, const double* ph, const double* mh,
                        const double* origin, double* x1, double* x2) {
  double v[2], xHalf[2];
  interp_global(m, 2, p1, origin, v);
  xHalf[0] = origin[0] - 0.5 * dt * v[0];
  xHalf[1] = origin[1] - 0.5 * dt * v[1];
  sl_periodic_update(m, xHalf);
  interp_global(m, 2, ph, xHalf, v);
  x1[0] = origin[0] - dt * v[0];
  x1[1] = origin[1] - dt * v[1];
  sl_periodic_update(m, x1);
  interp_global(m, 2, vel, x1, v);
  xHalf[0] = x1[0] - 0.5 * dt * v[0];
  xHalf[1] = x1[1] - 0.5 * dt * v[1];
  sl_periodic_update(m, xHalf);
  interp_global(m, 2, mh, xHalf, v);
  x2[0] = x1[0] - dt * v[0];
  x2[1] = x1[1] - dt * v[1];
  sl_periodic_update(m, x2);
}

typedef struct {
  const or_mesh* m;
  int ndofs;
  const double *field, *vel, *field_prev, *p1, *ph, *mh;
  double dt;
  double* out;
} advect_ctx;
static void advect_range(void* vctx, long b, long e, int t) {
  (void)t;
  advect_ctx* c = (advect_ctx*)vctx;
  const or_mesh* m = c->m;
  int ndofs = c->ndofs;
  const double *field = c->field, *vel = c->vel, *field_prev = c->field_prev;
  const double *p1 = c->p1, *ph = c->ph, *mh = c->mh;
  double dt = c->dt, *out = c->out;
  for (long n = b; n < e; n++) {
    double val[4], val2[4];
    const double* origin = m->verts + 2 * n;
    if (!field_prev) {
      double c[2];
      integrate_rk2(m, dt, vel, vel, origin, c);
      interp_global(m, ndofs, field, c, val);
      for (int d = 0; d < ndofs; d++) out[(size_t)n * ndofs + d] = val[d];
    } else {
      double x1[2], x2[2];
      trajectory2(m, dt, vel, p1, ph, mh, origin, x1, x2);
      interp_global(m, ndofs, field, x1, val);
      interp_global(m, ndofs, field_prev, x2, val2);
      for (int d = 0; d < ndofs; d++) out[(size_t)n * ndofs + d] = 2.0 * val[d] - 0.5 * val2[d];
    }
  }
}

/* src/base/Advector.cpp:181-246 (FirstOrder / SecondOrder): every vertex,
 * periodic duplicates included, then Field::PeriodicUpdate. */
int or_advect(const or_mesh* m, int ndofs, const double* field, const double* vel,
              const double* field_prev, const double* vel_prev, double dt,
              double* out, int nthreads) {
  if (m->N < 3) return -1;
  int nv = m->nVertsTotal;
  double *p1 = NULL, *ph = NULL, *mh = NULL;
  if (field_prev) {
    p1 = (double*)malloc(sizeof(double) * 2 * nv);
    ph = (double*)malloc(sizeof(double) * 2 * nv);
    mh = (double*)malloc(sizeof(double) * 2 * nv);
    extrapolate(nv, vel, vel_prev, p1, ph, mh);
  }
  advect_ctx ctx = {m, ndofs, field, vel, field_prev, p1, ph, mh, dt, out};
  par_for(nthreads, nv, advect_range, &ctx);
  if (m->periodic[0] || m->periodic[1]) or_periodic_update(m, ndofs, out);
  free(p1);
  free(ph);
  free(mh);
  return 0;
}

void or_departure_first(const or_mesh* m, const double* vel, double dt, double* dep,
                        int* el) {
  for (int n = 0; n < m->nVertsTotal; n++) {
    integrate_rk2(m, dt, vel, vel, m->verts + 2 * n, dep + 2 * n);
    el[n] = get_el(m, dep + 2 * n);
  }
}
void or_departure_second(const or_mesh* m, const double* vel, const double* vel_prev,
                         double dt, double* x1, int* el1, double* x2, int* el2) {
  int nv = m->nVertsTotal;
  double* p1 = (double*)malloc(sizeof(double) * 2 * nv);
  double* ph = (double*)malloc(sizeof(double) * 2 * nv);
  double* mh = (double*)malloc(sizeof(double) * 2 * nv);
  extrapolate(nv, vel, vel_prev, p1, ph, mh);
  for (int n = 0; n < nv; n++) {
    trajectory2(m, dt, vel, p1, ph, mh, m->verts + 2 * n, x1 + 2 * n, x2 + 2 * n);
    el1[n] = get_el(m, x1 + 2 * n);
    el2[n] = get_el(m, x2 + 2 * n);
  }
  free(p1);
  free(ph);
  free(mh);
}

/* ------------------------------------------------------------ gradients --
 * src/base/Legendre.cpp:187-223 (ShapeFuncDerivsAtCoord) and
 * src/base/Mesh.cpp:252-285 (global derivatives through the numerical
 * Jacobian), as used by Field::InterpDerivsGlobal (src/base/Field.cpp:96-118). */
static void jac_from_derivs(const or_mesh* m, int el, const double* g0,
                            const double* g1, double J[2][2], double* det) {
  int nodes[(MAXN + 1) * (MAXN + 1)];
  el_nodes(m, el, nodes);
  J[0][0] = J[0][1] = J[1][0] = J[1][1] = 0.0;
  for (int k = 0; k < m->nn; k++) {
    const double* v = m->verts + 2 * nodes[k];
    J[0][0] += g0[k] * v[0];
    J[0][1] += g0[k] * v[1];
    J[1][0] += g1[k] * v[0];
    J[1][1] += g1[k] * v[1];
  }
  *det = J[0][0] * J[1][1] - J[0][1] * J[1][0];
}
static void global_derivs(const or_mesh* m, int el, const double* g0, const double* g1,
                          double* gx, double* gy, double* det) {
  double J[2][2], temp;
  jac_from_derivs(m, el, g0, g1, J, det);
  temp = J[0][0];
  J[0][0] = J[1][1] / (*det);
  J[1][1] = temp / (*det);
  J[0][1] = -J[0][1] / (*det);
  J[1][0] = -J[1][0] / (*det);
  for (int k = 0; k < m->nn; k++) {
    double t = 0.0;
    t += g0[k] * J[0][0];
    t += g1[k] * J[0][1];
    gx[k] = t;
    t = 0.0;
    t += g0[k] * J[1][0];
    t += g1[k] * J[1][1];
    gy[k] = t;
  }
}
static void shape_derivs_at(const or_mesh* m, const double* c, double* g0, double* g1) {
  int N = m->N, xi, yi;
  for (int pt = 0; pt < m->nn; pt++) {
    int xj = pt % (N + 1), yj = pt / (N + 1);
    double Nx, Ny, GNx, GNy, a, b, cc;
    if (is_root(m, c[0], &xi)) {
      Nx = (xi == xj) ? 1.0 : 0.0;
      GNx = m->dC[xi * (N + 1) + xj];
    } else {
      double aj = m->abcissa[xj];
      Nx = -((1.0 - c[0] * c[0]) / (N * (N + 1) * jac_eval(N, m->Pc, aj) * (c[0] - aj))) *
           jac_deriv(N, m->Pc, c[0]);
      a = c[0] * c[0] + 1.0 - 2.0 * c[0] * aj;
      b = (1.0 - c[0] * c[0]) * (c[0] - aj);
      cc = N * (N + 1) * (c[0] - aj) * (c[0] - aj) * jac_eval(N, m->Pc, aj);
      GNx = (a * jac_deriv(N, m->Pc, c[0]) - b * jac_deriv2(N, m->Pc, c[0])) / cc;
    }
    if (is_root(m, c[1], &yi)) {
      Ny = (yi == yj) ? 1.0 : 0.0;
      GNy = m->dC[yi * (N + 1) + yj];
    } else {
      double aj = m->abcissa[yj];
      Ny = -((1.0 - c[1] * c[1]) / (N * (N + 1) * jac_eval(N, m->Pc, aj) * (c[1] - aj))) *
           jac_deriv(N, m->Pc, c[1]);
      a = c[1] * c[1] + 1.0 - 2.0 * c[1] * aj;
      b = (1.0 - c[1] * c[1]) * (c[1] - aj);
      cc = N * (N + 1) * (c[1] - aj) * (c[1] - aj) * jac_eval(N, m->Pc, aj);
      GNy = (a * jac_deriv(N, m->Pc, c[1]) - b * jac_deriv2(N, m->Pc, c[1])) / cc;
    }
    g0[pt] = GNx * Ny;
    g1[pt] = Nx * GNy;
  }
}
void or_interp_derivs_global(const or_mesh* m, const double* vals, const double* pts,
                             int npts, double* grad) {
  double g0[(MAXN + 1) * (MAXN + 1)], g1[(MAXN + 1) * (MAXN + 1)];
  double gx[(MAXN + 1) * (MAXN + 1)], gy[(MAXN + 1) * (MAXN + 1)];
  int nodes[(MAXN + 1) * (MAXN + 1)];
  for (int k = 0; k < npts; k++) {
    double l[2], det;
    int el = global_to_local(m, pts + 2 * k, l);
    el_nodes(m, el, nodes);
    shape_derivs_at(m, l, g0, g1);
    global_derivs(m, el, g0, g1, gx, gy, &det);
    double dx = 0.0, dy = 0.0;
    for (int q = 0; q < m->nn; q++) {
      dx += gx[q] * vals[nodes[q]];
      dy += gy[q] * vals[nodes[q]];
    }
    grad[2 * k] = dx;
    grad[2 * k + 1] = dy;
  }
}

/* ---------------------------------------------------------------- BCs -- */
/* src/base/BCs.cpp:36-195 (scalar constructor) and :371-389 (IsBCNode). */
int or_bcs_maps(const or_mesh* m, int bottom, int top, int left, int right,
                int* f2v, int* v2f) {
  int bB = bottom != 0, bT = top != 0, bL = left != 0, bR = right != 0;
  int nx = m->nVerts[0], ny = m->nVerts[1], nv = m->nVertsTotal, size = 0;
  if ((bB || bT) && m->periodic[1]) return -1;
  if ((bL || bR) && m->periodic[0]) return -1;
  if (m->periodic[0]) bR = 1;
  if (m->periodic[1]) bT = 1;
  if (bB) size += nx;
  if (bT || m->periodic[1]) size += nx;
  if (bL) size += ny;
  if (bR || m->periodic[0]) size += ny;
  if (bB && bL) size--;
  if (bB && bR) size--;
  if (bT && bL) size--;
  if (bT && bR) size--;
  int vec = 0;
#define ISBC(t0, t1) ((bB && (t1) == 0) || (bT && (t1) == ny - 1) || (bL && (t0) == 0) || (bR && (t0) == nx - 1))
  int both = (!m->periodic[0] && !m->periodic[1]) || (m->periodic[0] && m->periodic[1]);
  if (!both && !m->periodic[0]) return -1; /* periodic in y only: not built by the reference */
  for (int f = 0; f < nv; f++) {
    int t0 = f % nx, t1 = f / nx;
    if (!ISBC(t0, t1)) {
      v2f[vec] = f;
      f2v[f] = vec;
      vec++;
      continue;
    }
    if (both) {
      if (m->periodic[0] && m->periodic[1] && f == nv - 1)
        f2v[f] = 0;
      else if (m->periodic[0] && t0 == nx - 1)
        f2v[f] = t1 * (nx - 1);
      else if (m->periodic[1] && t1 == ny - 1)
        f2v[f] = t0;
      else
        f2v[f] = -1;
    } else if (bT && bB) {
      if (t1 == 0 || t1 == ny - 1)
        f2v[f] = -1;
      else if (t0 == nx - 1)
        f2v[f] = (t1 - 1) * (nx - 1);
      else
        return -1;
    } else if (bT) {
      if (t1 == ny - 1)
        f2v[f] = -1;
      else if (t0 == nx - 1)
        f2v[f] = t1 * (nx - 1);
      else
        return -1;
    } else {
      if (t0 == nx - 1)
        f2v[f] = t1 * (nx - 1);
      else
        return -1;
    }
  }
#undef ISBC
  if (vec != nv - size) return -1;
  return vec;
}

/* ------------------------------------------------------ element matrices --
 * src/base/Legendre.cpp:171-184 (reference derivatives at a GLL point),
 * src/base/Mesh.cpp:183-198 (DetJac), :217-250 (ShapeFuncDerivs). */
static void ref_derivs_at_pt(const or_mesh* m, int pt, double* g0, double* g1) {
  int N = m->N, xi = pt % (N + 1), yi = pt / (N + 1);
  for (int q = 0; q < m->nn; q++) {
    int xj = q % (N + 1), yj = q / (N + 1);
    g0[q] = (yi == yj) ? m->dC[xi * (N + 1) + xj] : 0.0;
    g1[q] = (xi == xj) ? m->dC[yi * (N + 1) + yj] : 0.0;
  }
}

/* MassMatrix(cMass) then Laplacian(cLap), accumulated into M in the order
 * HelmholtzEqn adds them (src/linsys/HelmholtzEqn.cpp:96-97); MassMatrix is
 * src/base/Operator.cpp:157-177, Laplacian :63-84 with detJac forced to 1
 * at :72 unless quirk == 0. */
void or_element_matrix(const or_mesh* m, int el, double cMass, double cLap,
                       int quirk, double* M) {
  int nn = m->nn, N = m->N;
  double g0[(MAXN + 1) * (MAXN + 1)], g1[(MAXN + 1) * (MAXN + 1)];
  double gx[(MAXN + 1) * (MAXN + 1)], gy[(MAXN + 1) * (MAXN + 1)];
  memset(M, 0, sizeof(double) * nn * nn);
  if (cMass != 0.0) {
    for (int pt = 0; pt < nn; pt++) {
      double weight = m->weights[pt % (N + 1)] * m->weights[pt / (N + 1)];
      double J[2][2], det;
      ref_derivs_at_pt(m, pt, g0, g1);
      jac_from_derivs(m, el, g0, g1, J, &det);
      for (int r = 0; r < nn; r++)
        for (int c = 0; c < nn; c++) {
          double Nr = (r == pt) ? 1.0 : 0.0, Nc = (c == pt) ? 1.0 : 0.0;
          M[r * nn + c] += det * weight * cMass * Nr * Nc;
        }
    }
  }
  if (cLap != 0.0) {
    for (int pt = 0; pt < nn; pt++) {
      double weight = m->weights[pt % (N + 1)] * m->weights[pt / (N + 1)];
      double det;
      ref_derivs_at_pt(m, pt, g0, g1);
      global_derivs(m, el, g0, g1, gx, gy, &det);
      if (quirk) det = 1.0;
      double w = det * weight * cLap;
      for (int r = 0; r < nn; r++)
        for (int c = 0; c < nn; c++) M[r * nn + c] += w * (gx[r] * gx[c] + gy[r] * gy[c]);
    }
  }
}

/* ------------------------------------------------------------------ SVV --
 * Spectral vanishing viscosity element matrix, restated literally from
 * src/base/SVV.cpp:120-176 (AssembleElement) with the modal basis of
 * src/base/Legendre.cpp:307-335 (ModalBasis: (1+x)/2, (1-x)/2, then
 * (1-x^2)/4 P_{i-2}^{(1,1)}) and the dense helpers of src/base/LinAlg.cpp
 * (Tran, Mult, Inv; the inverse here is Gauss-Jordan with partial pivoting,
 * equal to the reference's full-pivoting one up to rounding). Adds
 * constant*(Lxx + Lyy) to M; Lyy is formed from MinvQMDx exactly as the
 * reference forms it. */
static void svv_mult(const double* A, const double* B, double* C, int n) {
  for (int i = 0; i < n * n; i++) C[i] = 0.0;
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++)
      for (int k = 0; k < n; k++) C[i * n + j] += A[i * n + k] * B[k * n + j];
}
static void svv_tran(const double* A, double* At, int n) {
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) At[j * n + i] = A[i * n + j];
}
static int svv_inv(const double* A, double* Ainv, int n) {
  double* a = (double*)malloc(sizeof(double) * n * n);
  memcpy(a, A, sizeof(double) * n * n);
  for (int i = 0; i < n * n; i++) Ainv[i] = 0.0;
  for (int i = 0; i < n; i++) Ainv[i * n + i] = 1.0;
  for (int c = 0; c < n; c++) {
    int p = c;
    for (int r = c + 1; r < n; r++)
      if (fabs(a[r * n + c]) > fabs(a[p * n + c])) p = r;
    if (a[p * n + c] == 0.0) {
      free(a);
      return -1;
    }
    if (p != c)
      for (int k = 0; k < n; k++) {
        double t = a[c * n + k];
        a[c * n + k] = a[p * n + k];
        a[p * n + k] = t;
        t = Ainv[c * n + k];
        Ainv[c * n + k] = Ainv[p * n + k];
        Ainv[p * n + k] = t;
      }
    const double inv = 1.0 / a[c * n + c];
    for (int k = 0; k < n; k++) {
      a[c * n + k] *= inv;
      Ainv[c * n + k] *= inv;
    }
    for (int r = 0; r < n; r++) {
      if (r == c) continue;
      const double f = a[r * n + c];
      if (f == 0.0) continue;
      for (int k = 0; k < n; k++) {
        a[r * n + k] -= f * a[c * n + k];
        Ainv[r * n + k] -= f * Ainv[c * n + k];
      }
    }
  }
  free(a);
  return 0;
}
/* modal[i][0..N]: monomial coefficients of modal basis function i. */
static void svv_modal_basis(int N, double* modal) {
  double Pn[MAXN + 1][MAXN + 2];
  memset(Pn, 0, sizeof(Pn));
  memset(modal, 0, sizeof(double) * (N + 1) * (N + 1));
  Pn[0][0] = 1.0;
  if (N >= 1) Pn[1][1] = 2.0;
  for (int i = 2; i <= N; i++) jac_gen(i, 1.0, Pn[i - 1], i - 1, Pn[i - 2], i - 2, Pn[i]);
  modal[0 * (N + 1) + 0] = +0.5;
  modal[0 * (N + 1) + 1] = +0.5;
  modal[1 * (N + 1) + 0] = +0.5;
  modal[1 * (N + 1) + 1] = -0.5;
  for (int i = 2; i <= N; i++)
    for (int j = 0; j < i - 1; j++) {
      modal[i * (N + 1) + j] += 0.25 * Pn[i - 2][j];
      modal[i * (N + 1) + j + 2] -= 0.25 * Pn[i - 2][j];
    }
}
/* Jacobi::EvalTotal of a degree-n coefficient array. */
static double svv_eval_total(int n, const double* c, double x) {
  double p = 0.0;
  for (int i = n; i >= 0; i--) p += c[i] * pow(x, i);
  return p;
}
int or_svv_element(const or_mesh* m, int el, double constant, int mN, double* M) {
  const int N = m->N, nn = m->nn, n1 = N + 1;
  const size_t sz = sizeof(double) * nn * nn;
  double *Q = calloc(1, sz), *W = calloc(1, sz), *Lxx = calloc(1, sz), *Lyy = calloc(1, sz),
         *B = calloc(1, sz), *Bt = calloc(1, sz), *BtW = calloc(1, sz), *BtWB = calloc(1, sz),
         *BtWBinv = calloc(1, sz), *Mm = calloc(1, sz), *Minv = calloc(1, sz),
         *Dx = calloc(1, sz), *Dy = calloc(1, sz), *MinvQ = calloc(1, sz), *MinvQM = calloc(1, sz),
         *MinvQMDx = calloc(1, sz), *MinvQMDy = calloc(1, sz), *MinvQMDxt = calloc(1, sz),
         *MinvQMDyt = calloc(1, sz), *MinvQMDxtW = calloc(1, sz), *MinvQMDytW = calloc(1, sz);
  double modal[(MAXN + 1) * (MAXN + 1)];
  double g0[(MAXN + 1) * (MAXN + 1)], g1[(MAXN + 1) * (MAXN + 1)];
  svv_modal_basis(N, modal);
  int rc = 0;
  for (int i = 0; i < nn; i++) {
    const int ix = i / n1, iy = i % n1; /* GetRowCol(i, &ix, &iy, N+1) */
    const double weight = m->weights[i % n1] * m->weights[i / n1];
    double J[2][2], detJac;
    ref_derivs_at_pt(m, i, g0, g1); /* el->ShapeFuncDerivs(i) */
    jac_from_derivs(m, el, g0, g1, J, &detJac);
    for (int j = 0; j < nn; j++) {
      const int jx = j / n1, jy = j % n1;
      const int djx = jx < 2 ? 1 : jx, djy = jy < 2 ? 1 : jy; /* modal degree */
      B[i * nn + j] = svv_eval_total(djx, modal + jx * n1, m->abcissa[ix]) *
                      svv_eval_total(djy, modal + jy * n1, m->abcissa[iy]);
      W[i * nn + j] = Q[i * nn + j] = 0.0;
      if (i == j) {
        W[i * nn + j] = detJac * weight;
        if (jx > mN && jy > mN) {
          double qExpX = -1.0 * ((double)(N - jx) * (N - jx)) / ((mN - jx) * (mN - jx));
          double qExpY = -1.0 * ((double)(N - jy) * (N - jy)) / ((mN - jy) * (mN - jy));
          Q[i * nn + j] = sqrt(exp(qExpX + qExpY));
        }
      }
      Dx[i * nn + j] = g0[j];
      Dy[i * nn + j] = g1[j];
    }
  }
  svv_tran(B, Bt, nn); /* (the reference's Dxt, Dyt are never used) */
  svv_mult(Bt, W, BtW, nn);
  svv_mult(BtW, B, BtWB, nn);
  if (svv_inv(BtWB, BtWBinv, nn)) rc = -1;
  svv_mult(BtWBinv, BtW, Mm, nn);
  if (!rc && svv_inv(Mm, Minv, nn)) rc = -1;
  if (!rc) {
    svv_mult(Minv, Q, MinvQ, nn);
    svv_mult(MinvQ, Mm, MinvQM, nn);
    svv_mult(MinvQM, Dx, MinvQMDx, nn);
    svv_mult(MinvQM, Dy, MinvQMDy, nn);
    svv_tran(MinvQMDx, MinvQMDxt, nn);
    svv_tran(MinvQMDy, MinvQMDyt, nn);
    svv_mult(MinvQMDxt, W, MinvQMDxtW, nn);
    svv_mult(MinvQMDyt, W, MinvQMDytW, nn);
    svv_mult(MinvQMDxtW, MinvQMDx, Lxx, nn);
    svv_mult(MinvQMDxtW, MinvQMDx, Lyy, nn); /* as the reference: from MinvQMDx */
    for (int r = 0; r < nn; r++)
      for (int c = 0; c < nn; c++) M[r * nn + c] += constant * (Lxx[r * nn + c] + Lyy[r * nn + c]);
  }
  double* all[] = {Q, W, Lxx, Lyy, B, Bt, BtW, BtWB, BtWBinv, Mm, Minv, Dx, Dy, MinvQ, MinvQM,
                   MinvQMDx, MinvQMDy, MinvQMDxt, MinvQMDyt, MinvQMDxtW, MinvQMDytW};
  for (size_t k = 0; k < sizeof(all) / sizeof(all[0]); k++) free(all[k]);
  return rc;
}

/* src/base/RHSOp.cpp:31-50 (FieldRHS, constant 1): at GLL points the
 * interpolation snaps to the nodal value and the shape functions are a
 * Kronecker delta, so each node gets detJ*w*f plus zeros. */
void or_field_rhs_element(const or_mesh* m, const double* vals, int el, double* rhs) {
  int nn = m->nn, N = m->N;
  int nodes[(MAXN + 1) * (MAXN + 1)];
  double g0[(MAXN + 1) * (MAXN + 1)], g1[(MAXN + 1) * (MAXN + 1)];
  el_nodes(m, el, nodes);
  memset(rhs, 0, sizeof(double) * nn);
  for (int pt = 0; pt < nn; pt++) {
    double weight = m->weights[pt % (N + 1)] * m->weights[pt / (N + 1)];
    double J[2][2], det;
    ref_derivs_at_pt(m, pt, g0, g1);
    jac_from_derivs(m, el, g0, g1, J, &det);
    double f = 0.0;
    for (int k = 0; k < nn; k++) f += ((k == pt) ? 1.0 : 0.0) * vals[nodes[k]];
    double w = det * weight * 1.0;
    for (int k = 0; k < nn; k++) rhs[k] += w * f * ((k == pt) ? 1.0 : 0.0);
  }
}

/* ----------------------------------------------------- global assembly --
 * src/base/Matrix.cpp:63-149: element matrices scattered with ADD_VALUES
 * into the unknowns (Dirichlet rows/columns, map -1, dropped), explicit zeros
 * kept, and the Dirichlet lifting rhs -= M[:,D] u_D added per element. */
static int cmp_int(const void* a, const void* b) {
  int x = *(const int*)a, y = *(const int*)b;
  return (x > y) - (x < y);
}
or_csr* or_assemble(const or_mesh* m, const int* f2v, int ng, double cMass,
                    double cLap, int quirk, const double* sol_vals) {
  return or_assemble_svv(m, f2v, ng, cMass, cLap, quirk, sol_vals, 0.0, 0);
}
/* HelmholtzEqn's operators in its order (src/linsys/HelmholtzEqn.cpp:74-76):
 * mass, Laplacian, then SVV(svvConstant, svvCutoff) when svvCutoff != 0. */
or_csr* or_assemble_svv(const or_mesh* m, const int* f2v, int ng, double cMass,
                        double cLap, int quirk, const double* sol_vals, double svvConstant,
                        int svvCutoff) {
  int nn = m->nn;
  int nodes[(MAXN + 1) * (MAXN + 1)], rows[(MAXN + 1) * (MAXN + 1)];
  /* pattern: for each row the set of columns reached by any element */
  int* cnt = (int*)calloc(ng + 1, sizeof(int));
  for (int el = 0; el < m->nElsTotal; el++) {
    el_nodes(m, el, nodes);
    for (int r = 0; r < nn; r++) rows[r] = f2v[nodes[r]];
    for (int r = 0; r < nn; r++)
      if (rows[r] >= 0)
        for (int c = 0; c < nn; c++)
          if (rows[c] >= 0) cnt[rows[r]]++;
  }
  or_csr* A = (or_csr*)calloc(1, sizeof(or_csr));
  A->n = ng;
  A->rowptr = (int*)malloc(sizeof(int) * (ng + 1));
  A->rowptr[0] = 0;
  for (int i = 0; i < ng; i++) A->rowptr[i + 1] = A->rowptr[i] + cnt[i];
  int* tmp = (int*)malloc(sizeof(int) * A->rowptr[ng]);
  int* fill = (int*)calloc(ng, sizeof(int));
  for (int el = 0; el < m->nElsTotal; el++) {
    el_nodes(m, el, nodes);
    for (int r = 0; r < nn; r++) rows[r] = f2v[nodes[r]];
    for (int r = 0; r < nn; r++)
      if (rows[r] >= 0)
        for (int c = 0; c < nn; c++)
          if (rows[c] >= 0) tmp[A->rowptr[rows[r]] + fill[rows[r]]++] = rows[c];
  }
  /* unique sorted columns per row */
  int nnz = 0;
  int* newptr = (int*)malloc(sizeof(int) * (ng + 1));
  newptr[0] = 0;
  for (int i = 0; i < ng; i++) {
    int b = A->rowptr[i], e = A->rowptr[i + 1];
    qsort(tmp + b, e - b, sizeof(int), cmp_int);
    int last = -1;
    for (int k = b; k < e; k++)
      if (tmp[k] != last) {
        tmp[nnz++] = tmp[k];
        last = tmp[k];
      }
    newptr[i + 1] = nnz;
  }
  free(A->rowptr);
  A->rowptr = newptr;
  A->nnz = nnz;
  A->col = (int*)malloc(sizeof(int) * (nnz > 0 ? nnz : 1));
  memcpy(A->col, tmp, sizeof(int) * nnz);
  A->val = (double*)calloc(nnz > 0 ? nnz : 1, sizeof(double));
  A->lift = (double*)calloc(ng > 0 ? ng : 1, sizeof(double));
  free(tmp);
  free(fill);
  free(cnt);
  double* M = (double*)malloc(sizeof(double) * nn * nn);
  double* rhs = (double*)malloc(sizeof(double) * nn);
  for (int el = 0; el < m->nElsTotal; el++) {
    or_element_matrix(m, el, cMass, cLap, quirk, M);
    if (svvCutoff) or_svv_element(m, el, svvConstant, svvCutoff, M);
    el_nodes(m, el, nodes);
    for (int r = 0; r < nn; r++) rows[r] = f2v[nodes[r]];
    for (int r = 0; r < nn; r++) {
      if (rows[r] < 0) continue;
      int b = A->rowptr[rows[r]], e = A->rowptr[rows[r] + 1];
      for (int c = 0; c < nn; c++) {
        if (rows[c] < 0) continue;
        int lo = b, hi = e - 1;
        while (lo < hi) {
          int mid = (lo + hi) / 2;
          if (A->col[mid] < rows[c]) lo = mid + 1; else hi = mid;
        }
        A->val[lo] += M[r * nn + c];
      }
    }
    if (!sol_vals) continue;
    int add = 0;
    memset(rhs, 0, sizeof(double) * nn);
    for (int c = 0; c < nn; c++)
      if (rows[c] == -1) {
        add = 1;
        for (int r = 0; r < nn; r++) rhs[r] -= sol_vals[nodes[c]] * M[r * nn + c];
      }
    if (add)
      for (int r = 0; r < nn; r++)
        if (rows[r] >= 0) A->lift[rows[r]] += rhs[r];
  }
  free(M);
  free(rhs);
  return A;
}
void or_csr_destroy(or_csr* A) {
  if (!A) return;
  free(A->rowptr);
  free(A->col);
  free(A->val);
  free(A->lift);
  free(A);
}
typedef struct { const or_csr* A; const double* x; double* y; } matvec_ctx;
static void matvec_range(void* vctx, long b, long e, int t) {
  (void)t;
  matvec_ctx* c = (matvec_ctx*)vctx;
  const or_csr* A = c->A;
  for (long i = b; i < e; i++) {
    double s = 0.0;
    for (int k = A->rowptr[i]; k < A->rowptr[i + 1]; k++) s += A->val[k] * c->x[A->col[k]];
    c->y[i] = s;
  }
}
void or_csr_matvec(const or_csr* A, const double* x, double* y, int nthreads) {
  matvec_ctx c = {A, x, y};
  par_for(nthreads, A->n, matvec_range, &c);
}

/* src/base/Vector.cpp:89-121 with FieldRHS (src/base/RHSOp.cpp:31-50). */
void or_assemble_rhs(const or_mesh* m, const int* f2v, int ng, const double* rhs_vals,
                     double* f) {
  int nn = m->nn;
  int nodes[(MAXN + 1) * (MAXN + 1)];
  double rhs[(MAXN + 1) * (MAXN + 1)];
  memset(f, 0, sizeof(double) * ng);
  for (int el = 0; el < m->nElsTotal; el++) {
    or_field_rhs_element(m, rhs_vals, el, rhs);
    el_nodes(m, el, nodes);
    for (int k = 0; k < nn; k++) {
      int v = f2v[nodes[k]];
      if (v >= 0) f[v] += rhs[k];
    }
  }
}

/* -------------------------------------------------- two-layer QG pieces --
 * DissipationRHS::AssembleElement (src/qg/TwoLayerQGEqn.cpp:435-463)
 * assembled by Vector::Assemble (src/base/Vector.cpp:89-121) into the
 * unknowns: at every GLL point of every element, detJ w q N + c rF t N
 * - c Ei omegaHat N - c rF tau_e N - c nu (dN/dx dW/dx + dN/dy dW/dy), with
 * c = detJ w constant, the point values by InterpLocal (the nodal values),
 * and the gradient of omegaHat by InterpDerivsGlobal at the point's global
 * coordinate (Mesh::LocalToGlobal, src/base/Mesh.cpp:178-181), i.e. in the
 * element GetEl picks there. */
void or_dissipation_rhs(const or_mesh* m, const int* f2v, int ng, double constant,
                        const double* field, const double* tau, const double* omega_hat,
                        const double* tau_e, double rF, double Ei, double nu, double* f) {
  int nn = m->nn, N = m->N;
  int nodes[(MAXN + 1) * (MAXN + 1)], nodes2[(MAXN + 1) * (MAXN + 1)];
  double g0[(MAXN + 1) * (MAXN + 1)], g1[(MAXN + 1) * (MAXN + 1)];
  double gx[(MAXN + 1) * (MAXN + 1)], gy[(MAXN + 1) * (MAXN + 1)];
  double h0[(MAXN + 1) * (MAXN + 1)], h1[(MAXN + 1) * (MAXN + 1)];
  double hx[(MAXN + 1) * (MAXN + 1)], hy[(MAXN + 1) * (MAXN + 1)];
  double rhs[(MAXN + 1) * (MAXN + 1)];
  memset(f, 0, sizeof(double) * ng);
  for (int el = 0; el < m->nElsTotal; el++) {
    el_nodes(m, el, nodes);
    memset(rhs, 0, sizeof(double) * nn);
    for (int pt = 0; pt < nn; pt++) {
      double weight = m->weights[pt % (N + 1)] * m->weights[pt / (N + 1)];
      double det, det2, l[2], gc[2], l2[2];
      ref_derivs_at_pt(m, pt, g0, g1);
      global_derivs(m, el, g0, g1, gx, gy, &det);
      double c = det * weight * constant;
      l[0] = m->abcissa[pt % (N + 1)];
      l[1] = m->abcissa[pt / (N + 1)];
      gc[0] = m->min[0] + (el % m->nEls[0]) * m->dx[0] + 0.5 * (l[0] + 1.0) * m->dx[0];
      gc[1] = m->min[1] + (el / m->nEls[0]) * m->dx[1] + 0.5 * (l[1] + 1.0) * m->dx[1];
      double q = 0.0, t = 0.0, w = 0.0, te = 0.0;
      for (int k = 0; k < nn; k++) {
        double Nk = (k == pt) ? 1.0 : 0.0;
        q += Nk * field[nodes[k]];
        t += Nk * tau[nodes[k]];
        w += Nk * omega_hat[nodes[k]];
        te += Nk * tau_e[nodes[k]];
      }
      int el2 = global_to_local(m, gc, l2);
      el_nodes(m, el2, nodes2);
      shape_derivs_at(m, l2, h0, h1);
      global_derivs(m, el2, h0, h1, hx, hy, &det2);
      double gW0 = 0.0, gW1 = 0.0;
      for (int k = 0; k < nn; k++) {
        gW0 += hx[k] * omega_hat[nodes2[k]];
        gW1 += hy[k] * omega_hat[nodes2[k]];
      }
      for (int k = 0; k < nn; k++) {
        double Nk = (k == pt) ? 1.0 : 0.0;
        rhs[k] += det * weight * q * Nk;
        rhs[k] += c * rF * t * Nk;
        rhs[k] -= c * Ei * w * Nk;
        rhs[k] -= c * rF * te * Nk;
        rhs[k] -= c * nu * (gx[k] * gW0 + gy[k] * gW1);
      }
    }
    for (int k = 0; k < nn; k++) {
      int v = f2v[nodes[k]];
      if (v >= 0) f[v] += rhs[k];
    }
  }
}

/* Diagonal of TwoLayerQGEqn::AssembleQMat's matrix (src/qg/TwoLayerQGEqn.cpp:
 * 354-394): MassMatrix(qi, qi, a) assembled over the unknowns; the GLL mass
 * matrix is diagonal, so this is the whole matrix (and its Dirichlet lifting
 * is zero). */
void or_mass_diag(const or_mesh* m, const int* f2v, int ng, double a, double* d) {
  int nn = m->nn, N = m->N;
  int nodes[(MAXN + 1) * (MAXN + 1)];
  double g0[(MAXN + 1) * (MAXN + 1)], g1[(MAXN + 1) * (MAXN + 1)];
  memset(d, 0, sizeof(double) * ng);
  for (int el = 0; el < m->nElsTotal; el++) {
    el_nodes(m, el, nodes);
    for (int pt = 0; pt < nn; pt++) {
      double weight = m->weights[pt % (N + 1)] * m->weights[pt / (N + 1)];
      double J[2][2], det;
      ref_derivs_at_pt(m, pt, g0, g1);
      jac_from_derivs(m, el, g0, g1, J, &det);
      int v = f2v[nodes[pt]];
      if (v >= 0) d[v] += det * weight * a;
    }
  }
}

/* ------------------------------------------------------------------ PCG --
 * PETSc KSPCG with PCJACOBI as SE runs it through
 * src/linsys/HelmholtzEqn.cpp:141-150 with -<prefix>ksp_type cg
 * -<prefix>pc_type jacobi (PETSc: third party, version unpinned). Zero
 * initial guess; convergence when the chosen residual norm falls to
 * max(rtol*|r0|, atol); sign checks for an indefinite matrix or
 * preconditioner as KSPCG does; a constant null space is removed from every
 * preconditioned residual (KSP_PCApply followed by MatNullSpaceRemove). */
typedef struct { const double *a, *b; double part[256]; } dot_ctx;
static void dot_range(void* vctx, long b, long e, int t) {
  dot_ctx* c = (dot_ctx*)vctx;
  double s = 0.0;
  for (long i = b; i < e; i++) s += c->a[i] * c->b[i];
  c->part[t] = s;
}
static double dot_det(const double* a, const double* b, int n, int nthreads) {
  /* fixed chunks summed in order: deterministic for a given thread count.
   * Vectors this small are not worth a thread each. */
  int nt = nthreads > 0 ? nthreads : 1;
  if (nt > 256) nt = 256;
  if ((long)n < 65536L * nt) nt = 1;
  dot_ctx c;
  c.a = a;
  c.b = b;
  par_for(nt, n, dot_range, &c);
  double s = 0.0;
  for (int t = 0; t < nt; t++) s += c.part[t];
  return s;
}
static void remove_const(double* v, int n) {
  double s = 0.0;
  for (int i = 0; i < n; i++) s += v[i];
  s /= n;
  for (int i = 0; i < n; i++) v[i] -= s;
}
int or_pcg(const or_csr* A, const double* b_in, double* x, double rtol, double atol,
           double dtol, int max_it, int norm_type, int remove_null_space, int nthreads,
           int* its_out, double* rnorm_out, double* rnorm0_out) {
  int n = A->n, reason = 0, i = 0;
  double *r = (double*)malloc(sizeof(double) * n), *z = (double*)malloc(sizeof(double) * n);
  double *p = (double*)malloc(sizeof(double) * n), *w = (double*)malloc(sizeof(double) * n);
  double* dinv = (double*)malloc(sizeof(double) * n);
  for (int k = 0; k < n; k++) {
    double d = 0.0;
    for (int q = A->rowptr[k]; q < A->rowptr[k + 1]; q++)
      if (A->col[q] == k) d = A->val[q];
    dinv[k] = (d != 0.0) ? 1.0 / d : 1.0;
  }
  memset(x, 0, sizeof(double) * n);
  memcpy(r, b_in, sizeof(double) * n);
#define PCAPPLY()                                       \
  do {                                                  \
    for (int k = 0; k < n; k++) z[k] = r[k] * dinv[k];  \
    if (remove_null_space) remove_const(z, n);          \
  } while (0)
  PCAPPLY();
  double dp, beta = 0.0, betaold = 0.0, dpi = 0.0, dpiold = 0.0, a, bcoef;
  if (norm_type == 0)
    dp = sqrt(dot_det(z, z, n, nthreads));
  else if (norm_type == 1)
    dp = sqrt(dot_det(r, r, n, nthreads));
  else {
    beta = dot_det(z, r, n, nthreads);
    dp = sqrt(fabs(beta));
  }
  if (norm_type != 2) beta = dot_det(z, r, n, nthreads);
  double rnorm0 = dp, ttol = rtol * rnorm0 > atol ? rtol * rnorm0 : atol;
  if (isnan(dp) || isinf(dp)) reason = -9;
  else if (dp <= ttol) reason = (dp < atol) ? 3 : 2;
  double rn = dp;
  while (!reason && i < max_it) {
    if (beta == 0.0) { reason = 3; break; }
    if (i > 0 && beta * betaold < 0.0) { reason = -8; break; }
    if (i == 0) {
      memcpy(p, z, sizeof(double) * n);
    } else {
      bcoef = beta / betaold;
      for (int k = 0; k < n; k++) p[k] = z[k] + bcoef * p[k];
    }
    dpiold = dpi;
    or_csr_matvec(A, p, w, nthreads);
    dpi = dot_det(p, w, n, nthreads);
    betaold = beta;
    if (dpi == 0.0 || (i > 0 && dpi * dpiold <= 0.0)) { reason = -10; break; }
    a = beta / dpi;
    for (int k = 0; k < n; k++) x[k] += a * p[k];
    for (int k = 0; k < n; k++) r[k] -= a * w[k];
    PCAPPLY();
    if (norm_type == 0)
      dp = sqrt(dot_det(z, z, n, nthreads));
    else if (norm_type == 1)
      dp = sqrt(dot_det(r, r, n, nthreads));
    else {
      beta = dot_det(z, r, n, nthreads);
      dp = sqrt(fabs(beta));
    }
    rn = dp;
    i++;
    if (isnan(dp) || isinf(dp)) { reason = -9; break; }
    if (dp <= ttol) { reason = (dp < atol) ? 3 : 2; break; }
    if (dp >= dtol * rnorm0) { reason = -4; break; }
    if (norm_type != 2) beta = dot_det(z, r, n, nthreads);
  }
#undef PCAPPLY
  if (!reason) reason = -3;
  if (its_out) *its_out = i;
  if (rnorm_out) *rnorm_out = rn;
  if (rnorm0_out) *rnorm0_out = rnorm0;
  free(r); free(z); free(p); free(w); free(dinv);
  return reason;
}

/* src/base/Vector.cpp:40-61 (scalar field, offset 0) */
void or_update_field(const or_mesh* m, const int* v2f, int ng, const double* x,
                     double* vals) {
  for (int k = 0; k < ng; k++) vals[v2f[k] % m->nVertsTotal] = x[k];
  if (m->periodic[0] || m->periodic[1]) or_periodic_update(m, 1, vals);
}

/* --------------------------------------------------------- diagnostics -- */
/* src/base/Field.cpp:181-200 */
double or_integrate(const or_mesh* m, const double* vals) {
  int N = m->N, nodes[(MAXN + 1) * (MAXN + 1)];
  double g0[(MAXN + 1) * (MAXN + 1)], g1[(MAXN + 1) * (MAXN + 1)];
  double xtot = 0.0;
  for (int el = 0; el < m->nElsTotal; el++) {
    el_nodes(m, el, nodes);
    for (int pt = 0; pt < m->nn; pt++) {
      double weight = m->weights[pt % (N + 1)] * m->weights[pt / (N + 1)];
      double J[2][2], det;
      ref_derivs_at_pt(m, pt, g0, g1);
      jac_from_derivs(m, el, g0, g1, J, &det);
      xtot += det * weight * vals[nodes[pt]];
    }
  }
  return xtot;
}
/* src/base/Utils.cpp:232-254 with the analytic field interpolated at the
 * element's own quadrature points. */
double or_field_error(const or_mesh* m, const double* numeric, const double* analytic,
                      int normalise) {
  int N = m->N, nodes[(MAXN + 1) * (MAXN + 1)];
  double g0[(MAXN + 1) * (MAXN + 1)], g1[(MAXN + 1) * (MAXN + 1)];
  double errSq = 0.0, normSq = 0.0;
  for (int el = 0; el < m->nElsTotal; el++) {
    double elErr = 0.0, elNorm = 0.0;
    el_nodes(m, el, nodes);
    for (int pt = 0; pt < m->nn; pt++) {
      double lc[2] = {m->abcissa[pt % (N + 1)], m->abcissa[pt / (N + 1)]}, gc[2], a;
      double weight = m->weights[pt % (N + 1)] * m->weights[pt / (N + 1)];
      double J[2][2], det;
      ref_derivs_at_pt(m, pt, g0, g1);
      jac_from_derivs(m, el, g0, g1, J, &det);
      gc[0] = m->min[0] + (el % m->nEls[0]) * m->dx[0] + 0.5 * (lc[0] + 1.0) * m->dx[0];
      gc[1] = m->min[1] + (el / m->nEls[0]) * m->dx[1] + 0.5 * (lc[1] + 1.0) * m->dx[1];
      interp_global(m, 1, analytic, gc, &a);
      double nv = numeric[nodes[pt]];
      elErr += det * weight * (nv - a) * (nv - a);
      elNorm += det * weight * a * a;
    }
    errSq += elErr;
    normSq += elNorm;
  }
  return normalise ? sqrt(errSq / normSq) : sqrt(errSq);
}
/* src/base/Utils.cpp:23-40 */
double or_calc_time_step(const or_mesh* m, const double* vel, double courant) {
  double dx = m->dx[0], dy = m->dx[1], minSep = (dx < dy) ? dx : dy, maxSq = 0.0;
  for (int v = 0; v < m->nVertsTotal; v++) {
    double s = vel[2 * v] * vel[2 * v] + vel[2 * v + 1] * vel[2 * v + 1];
    if (s > maxSq) maxSq = s;
  }
  return courant * minSep / sqrt(maxSq);
}
