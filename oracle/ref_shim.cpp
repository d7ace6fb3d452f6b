// C-ABI shim over the reference's own compiled src/base classes.
//
// TEST INFRASTRUCTURE ONLY. This file is compiled together with the
// reference's unmodified src/base sources (see oracle/Makefile) into
// oracle/_ref/libseref.so. Only tests/, the smoke check and bench.py's CPU
// baseline load it, and only as the checker; the product never does.
//
// Each entry point drives the reference classes exactly as the reference's
// own callers do, so that the outputs are the reference's own numbers:
//   Legendre tables     src/base/Legendre.cpp:15-125
//   Mesh / GetEl        src/base/Mesh.cpp:17-84, 109-176
//   BCs maps            src/base/BCs.cpp:14-195
//   element matrices    src/base/Operator.cpp:63-84 (Laplacian), 157-177 (MassMatrix),
//                       src/base/SVV.cpp:50-176 (SVV)
//   FieldRHS            src/base/RHSOp.cpp:31-50
//   Advector            src/base/Advector.cpp:136-274
//   InterpDerivsGlobal  src/base/Field.cpp:96-118
//   Integrate           src/base/Field.cpp:181-200
#include <cmath>
#include <cstdio>
#include <cstring>
#include <iostream>
#include <sstream>
#include <string>

// The reference declares the trajectory integrator and a few tables private;
// exposing them lets the shim call the reference's own code for departure
// points instead of restating it.
#define private public
#include "QuadPoint.h"
#include "LinAlg.h"
#include "Jacobi.h"
#include "Element.h"
#include "Legendre.h"
#include "Mesh.h"
#include "BCs.h"
#include "Field.h"
#include "Operator.h"
#include "RHSOp.h"
#include "Advector.h"
#include "SVV.h"
#undef private

namespace {
// The reference prints progress lines to stdout; keep test output clean.
struct Quiet {
  std::streambuf* old;
  std::ostringstream sink;
  Quiet() { old = std::cout.rdbuf(sink.rdbuf()); }
  ~Quiet() { std::cout.rdbuf(old); }
};

void load(Field* f, const double* vals) {
  for (int v = 0; v < f->mesh->nVertsTotal; v++)
    for (int d = 0; d < f->nDofs; d++) f->vals[v][d] = vals[v * f->nDofs + d];
}
void store(const Field* f, double* vals) {
  for (int v = 0; v < f->mesh->nVertsTotal; v++)
    for (int d = 0; d < f->nDofs; d++) vals[v * f->nDofs + d] = f->vals[v][d];
}
}  // namespace

extern "C" {

// GLL tables of order N: abcissa[N+1], weights[N+1], dCij[(N+1)^2] (row =
// point, col = basis) and P_N evaluated at each node, Pj[N+1].
void ref_gll(int N, double* abcissa, double* weights, double* dCij, double* Pj) {
  Legendre el(N);
  for (int i = 0; i <= N; i++) {
    abcissa[i] = el.abcissa[i];
    weights[i] = el.weights[i];
    Pj[i] = el.P->Eval(el.abcissa[i]);
  }
  for (int i = 0; i < (N + 1) * (N + 1); i++) dCij[i] = el.dCij[i];
}

// Legendre::ShapeFuncsAtCoord at npts local coordinates (xi, eta) pairs.
void ref_shape_funcs_at(int N, const double* coords, int npts, double* Ni) {
  Legendre el(N);
  int nn = (N + 1) * (N + 1);
  for (int k = 0; k < npts; k++) {
    double c[2] = {coords[2 * k], coords[2 * k + 1]};
    double* out = el.ShapeFuncsAtCoord(c);
    std::memcpy(Ni + (size_t)k * nn, out, sizeof(double) * nn);
  }
}

void* ref_mesh_create(int nx, int ny, int N, double x0, double y0, double x1,
                      double y1, int perx, int pery) {
  int nEls[2] = {nx, ny};
  double mn[2] = {x0, y0}, mx[2] = {x1, y1};
  bool per[2] = {perx != 0, pery != 0};
  return new Mesh("mesh", nEls, "legendre", N, mn, mx, per);
}
void ref_mesh_destroy(void* m) { delete (Mesh*)m; }
int ref_mesh_nverts(void* m) { return ((Mesh*)m)->nVertsTotal; }
void ref_mesh_verts(void* m, double* out) {
  Mesh* mesh = (Mesh*)m;
  for (int v = 0; v < mesh->nVertsTotal; v++) {
    out[2 * v] = mesh->verts[v][0];
    out[2 * v + 1] = mesh->verts[v][1];
  }
}
// Mesh::GlobalToLocal for npts global points: element index and local coords.
void ref_global_to_local(void* m, const double* pts, int npts, int* el, double* lc) {
  Mesh* mesh = (Mesh*)m;
  for (int k = 0; k < npts; k++) {
    double g[2] = {pts[2 * k], pts[2 * k + 1]};
    double l[2];
    mesh->GlobalToLocal(g, &el[k], l);
    lc[2 * k] = l[0];
    lc[2 * k + 1] = l[1];
  }
}

void* ref_bcs_create(void* m, int bottom, int top, int left, int right) {
  return new BCs(bottom != 0, top != 0, left != 0, right != 0, (Mesh*)m, 0);
}
void ref_bcs_destroy(void* b) { delete (BCs*)b; }
// Number of vector unknowns (nVertsTotal - size[0]).
int ref_bcs_vecsize(void* b) {
  BCs* bcs = (BCs*)b;
  return bcs->mesh->nVertsTotal - bcs->size[0];
}
void ref_bcs_maps(void* b, int* field_to_vec, int* vec_to_field) {
  BCs* bcs = (BCs*)b;
  int nv = bcs->mesh->nVertsTotal, ng = nv - bcs->size[0];
  std::memcpy(field_to_vec, bcs->fieldToVecMap, sizeof(int) * nv);
  std::memcpy(vec_to_field, bcs->vecToFieldMap, sizeof(int) * ng);
}

// Element matrix of MassMatrix(cMass) + Laplacian(cLap) for element el, in
// the order HelmholtzEqn builds it (mass first, src/linsys/HelmholtzEqn.cpp:96-97).
void ref_element_matrix(void* m, int el, double cMass, double cLap, double* M) {
  Mesh* mesh = (Mesh*)m;
  Field f("f", mesh, 1, NULL);
  int nn = mesh->el->nNodes;
  std::memset(M, 0, sizeof(double) * nn * nn);
  MassMatrix mass("m", &f, &f, cMass);
  Laplacian lap("l", &f, &f, cLap);
  if (cMass != 0.0) mass.AssembleElement(el, M);
  if (cLap != 0.0) lap.AssembleElement(el, M);
}

// SVV(constant, mN) element matrix for element el of a scalar field (the
// operator HelmholtzEqn adds when svvCutoff != 0, src/linsys/HelmholtzEqn.cpp:71).
void ref_svv_element(void* m, int el, double constant, int mN, double* M) {
  Mesh* mesh = (Mesh*)m;
  Field f("f", mesh, 1, NULL);
  int nn = mesh->el->nNodes;
  std::memset(M, 0, sizeof(double) * nn * nn);
  SVV svv("s", &f, &f, constant, mN);
  svv.AssembleElement(el, M);
}

// FieldRHS (constant 1) element vector for element el of a scalar field.
void ref_field_rhs_element(void* m, const double* vals, int el, double* rhs) {
  Mesh* mesh = (Mesh*)m;
  Field f("f", mesh, 1, NULL);
  load(&f, vals);
  FieldRHS op("rhs", mesh, 1.0, &f);
  std::memset(rhs, 0, sizeof(double) * mesh->el->nNodes);
  op.AssembleElement(el, rhs);
}

// Advector::Advect, first order (field_prev == NULL) or second order.
// field/vel are [nVertsTotal][ndofs] row-major; out receives fieldSL.
void ref_advect(void* m, int ndofs, const double* field, const double* vel,
                const double* field_prev, const double* vel_prev, double dt,
                double* out) {
  Quiet q;
  Mesh* mesh = (Mesh*)m;
  Field f("psi", mesh, ndofs, NULL), v("vel", mesh, 2, NULL);
  load(&f, field);
  load(&v, vel);
  if (field_prev) {
    Field fp("psiPrev", mesh, ndofs, NULL), vp("velPrev", mesh, 2, NULL);
    load(&fp, field_prev);
    load(&vp, vel_prev);
    Advector adv(&f, &v, &fp, &vp);
    adv.Advect(dt);
    store(adv.fieldSL, out);
  } else {
    Advector adv(&f, &v);
    adv.Advect(dt);
    store(adv.fieldSL, out);
  }
}

// First-order departure points of every vertex through the reference's own
// Advector::IntegrateRK2, and the element Mesh::GetEl assigns to each.
void ref_departure_first(void* m, const double* vel, double dt, double* dep, int* el) {
  Mesh* mesh = (Mesh*)m;
  Field f("psi", mesh, 1, NULL), v("vel", mesh, 2, NULL);
  load(&v, vel);
  Advector adv(&f, &v);
  for (int n = 0; n < mesh->nVertsTotal; n++) {
    double c[3];
    adv.IntegrateRK2(dt, &v, mesh->verts[n], c);
    dep[2 * n] = c[0];
    dep[2 * n + 1] = c[1];
    mesh->GetEl(c, &el[n]);
  }
}

// Field::InterpDerivsGlobal of a scalar field at npts global points:
// grad[2k] = d/dx, grad[2k+1] = d/dy.
void ref_interp_derivs_global(void* m, const double* vals, const double* pts,
                              int npts, double* grad) {
  Mesh* mesh = (Mesh*)m;
  Field f("psi", mesh, 1, NULL);
  load(&f, vals);
  double g0[2];
  double* gv[1] = {g0};
  for (int k = 0; k < npts; k++) {
    double c[2] = {pts[2 * k], pts[2 * k + 1]};
    f.InterpDerivsGlobal(c, gv);
    grad[2 * k] = g0[0];
    grad[2 * k + 1] = g0[1];
  }
}

// Field::InterpGlobal of an ndofs field at npts global points.
void ref_interp_global(void* m, int ndofs, const double* vals, const double* pts,
                       int npts, double* out) {
  Mesh* mesh = (Mesh*)m;
  Field f("psi", mesh, ndofs, NULL);
  load(&f, vals);
  for (int k = 0; k < npts; k++) {
    double c[3] = {pts[2 * k], pts[2 * k + 1], 0.0}, v[3];
    f.InterpGlobal(c, v);
    for (int d = 0; d < ndofs; d++) out[k * ndofs + d] = v[d];
  }
}

double ref_integrate(void* m, const double* vals) {
  Mesh* mesh = (Mesh*)m;
  Field f("psi", mesh, 1, NULL);
  load(&f, vals);
  return f.Integrate(0, false);
}

}  // extern "C"
