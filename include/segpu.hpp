/* segpu.hpp -- the reference's hot-path class signatures over the C-ABI of
 * segpu.h, header only. A caller of SE (src/qg, src/ns, src/sw, models/)
 * includes this header in place of the reference's Mesh.h, BCs.h, Field.h,
 * Advector.h, HelmholtzEqn.h and PoissonEqn.h (plus the QG and NS step
 * headers) and links libsegpu.so instead of those classes' objects.
 *
 * Field values live on the GPU. The reference's callers read and write
 * Field::vals (double**, one pointer per vertex); the shim keeps a host
 * mirror in the reference's layout that Upload()/Download() move, at the
 * points where the caller touches vals (after setting initial conditions,
 * before diagnostics or output). Code that stays on the GPU between steps
 * needs no copies. Every failing call throws std::runtime_error with the
 * library's message (the reference calls exit(1) on configuration errors).
 */
#ifndef SEGPU_HPP
#define SEGPU_HPP

#include <stdexcept>
#include <string>
#include <vector>

#include "segpu.h"

inline void se_ok(int rc) {
  if (rc) throw std::runtime_error(se_last_error());
}

/* Mesh(name, nEls, elType, N, min, max, periodic), src/base/Mesh.h:6 */
class Mesh {
 public:
  Mesh(std::string name, int nEls[2], std::string elType, int N, double min[2], double max[2],
       bool periodic[2])
      : name(name) {
    if (elType != "legendre") throw std::runtime_error("only legendre (GLL) elements");
    const int per[2] = {periodic[0], periodic[1]};
    se_ok(se_mesh_create(nEls, N, min, max, per, &h));
    se_ok(se_mesh_sizes(h, nVerts, &nVertsTotal));
  }
  ~Mesh() { se_mesh_destroy(h); }
  Mesh(const Mesh&) = delete;
  Mesh& operator=(const Mesh&) = delete;
  void Save() { se_ok(se_mesh_save(h, name.c_str())); }
  std::string name;
  int nVerts[2] = {0, 0}, nVertsTotal = 0;
  se_mesh* h = nullptr;
};

/* BCs(bottom, top, left, right, mesh, vecOffset), src/base/BCs.h:3 */
class BCs {
 public:
  BCs(bool bottom, bool top, bool left, bool right, Mesh* mesh, int vecOffset = 0) {
    if (vecOffset != 0) throw std::runtime_error("vecOffset != 0 is not supported");
    se_ok(se_bcs_create(mesh->h, bottom, top, left, right, &h));
  }
  ~BCs() { se_bcs_destroy(h); }
  BCs(const BCs&) = delete;
  BCs& operator=(const BCs&) = delete;
  int VecSize() const {
    int n = 0;
    se_ok(se_bcs_vec_size(h, &n));
    return n;
  }
  se_bcs* h = nullptr;
};

/* Field(name, mesh, nDofs, bcs) with public vals, src/base/Field.h:7-11 */
class Field {
 public:
  Field(std::string name, Mesh* mesh, int nDofs, BCs* bcs)
      : name(name), mesh(mesh), nDofs(nDofs), host((size_t)mesh->nVertsTotal * nDofs),
        vals(mesh->nVertsTotal) {
    se_ok(se_field_create(mesh->h, nDofs, bcs ? bcs->h : nullptr, &h));
    for (int i = 0; i < mesh->nVertsTotal; i++) vals[i] = &host[(size_t)i * nDofs];
  }
  ~Field() { se_field_destroy(h); }
  Field(const Field&) = delete;
  Field& operator=(const Field&) = delete;
  void Upload() { se_ok(se_field_upload(h, host.data())); }      // after writing vals
  void Download() { se_ok(se_field_download(h, host.data())); }  // before reading vals
  void Copy(Field* f) { se_ok(se_field_copy(h, f->h)); }
  double Integrate(int dof, bool average) {
    double r = 0.0;
    se_ok(se_field_integrate(h, dof, average, &r));
    return r;
  }
  void Save(int timeStep) { se_ok(se_field_save(h, name.c_str(), timeStep)); }
  void Read(int timeStep) { se_ok(se_field_read(h, name.c_str(), timeStep)); }
  std::string name;
  Mesh* mesh;
  int nDofs;
  std::vector<double> host;
  std::vector<double*> vals;
  se_field* h = nullptr;
};

/* Advector(field, velocity[, fieldPrev, velPrev]), Advect(dt) and the public
 * fieldSL, src/base/Advector.h:3-15. fieldSL is the advector's own device
 * field; wrap it with FieldSL() to read it on the host. */
class Advector {
 public:
  Advector(Field* f, Field* vel, Field* fPrev = nullptr, Field* velPrev = nullptr) {
    se_ok(se_advector_create(f->h, vel->h, fPrev ? fPrev->h : nullptr,
                             velPrev ? velPrev->h : nullptr, &h));
    se_ok(se_advector_field_sl(h, &fieldSL));
  }
  ~Advector() { se_advector_destroy(h); }
  Advector(const Advector&) = delete;
  Advector& operator=(const Advector&) = delete;
  void Advect(double dt) { se_ok(se_advect(h, dt)); }
  void DownloadSL(std::vector<double>& out, int nVertsTotal, int nDofs) {
    out.resize((size_t)nVertsTotal * nDofs);
    se_ok(se_field_download(fieldSL, out.data()));
  }
  se_field* fieldSL = nullptr;
  se_advector* h = nullptr;
};

/* Options of a solve: the reference reads -<prefix>ksp_* / pc_type from
 * PETSc's options database at every Solve; the shim takes the same string. */
inline se_solver_opts se_options(const std::string& prefix, const char* options) {
  se_solver_opts o;
  se_ok(se_solver_opts_default(&o));
  if (options && *options) se_ok(se_solver_opts_parse(&o, prefix.c_str(), options));
  return o;
}

/* HelmholtzEqn(sol, rhs, c, nu, dt, svvCutoff), Assemble(), Solve(prefix,
 * removeNullSpace), src/linsys/HelmholtzEqn.h:3-19. The reference never
 * checks convergence; neither does Solve (last() holds the statistics). */
class HelmholtzEqn {
 public:
  HelmholtzEqn(Field* sol, Field* rhs, double c, double nu, double dt, int svvCutoff) {
    se_solver_opts o = se_options("", nullptr);
    se_ok(se_helmholtz_create(sol->h, rhs ? rhs->h : nullptr, c, nu, dt, svvCutoff, &o, &h));
  }
  ~HelmholtzEqn() { se_linsys_destroy(h); }
  HelmholtzEqn(const HelmholtzEqn&) = delete;
  HelmholtzEqn& operator=(const HelmholtzEqn&) = delete;
  void Assemble() { se_ok(se_linsys_assemble(h)); }
  void Solve(std::string prefix, bool removeNullSpace, const char* options = "") {
    se_solver_opts o = se_options(prefix, options);
    se_ok(se_linsys_set_opts(h, &o));
    const int rc = se_linsys_solve(h, removeNullSpace ? 1 : 0, &stats);
    if (rc && rc != SE_ERR_NOT_CONVERGED) se_ok(rc);
  }
  const se_solve_stats& last() const { return stats; }
  se_linsys* h = nullptr;
  se_solve_stats stats = {};
};

/* PoissonEqn(sol, rhs, c), Solve(removeNullSpace), src/linsys/PoissonEqn.h:3-16
 * (options prefix "poisson_"). */
class PoissonEqn {
 public:
  PoissonEqn(Field* sol, Field* rhs, double c) {
    se_solver_opts o = se_options("", nullptr);
    se_ok(se_poisson_create(sol->h, rhs ? rhs->h : nullptr, c, &o, &h));
  }
  ~PoissonEqn() { se_linsys_destroy(h); }
  PoissonEqn(const PoissonEqn&) = delete;
  PoissonEqn& operator=(const PoissonEqn&) = delete;
  void Solve(bool removeNullSpace, const char* options = "") {
    se_solver_opts o = se_options("poisson_", options);
    se_ok(se_linsys_set_opts(h, &o));
    const int rc = se_linsys_solve(h, removeNullSpace ? 1 : 0, &stats);
    if (rc && rc != SE_ERR_NOT_CONVERGED) se_ok(rc);
  }
  const se_solve_stats& last() const { return stats; }
  se_linsys* h = nullptr;
  se_solve_stats stats = {};
};

/* TwoLayerQGEqn(psi1, omega1, psi2, omega2, F1, F2, beta, E2, r, nu, tau_e,
 * dt) and Solve(prev fields), src/qg/TwoLayerQGEqn.h. */
class TwoLayerQGEqn {
 public:
  TwoLayerQGEqn(Field* psi1, Field* omega1, Field* psi2, Field* omega2, double F1, double F2,
                double beta, double E2, double r, double nu, Field* tau_e, double dt,
                const char* options = "") {
    se_solver_opts o = se_options("helm_", options);
    se_ok(se_qg2_create(psi1->h, omega1->h, psi2->h, omega2->h, F1, F2, beta, E2, r, nu,
                        tau_e->h, dt, &o, &h));
  }
  ~TwoLayerQGEqn() { se_qg2_destroy(h); }
  TwoLayerQGEqn(const TwoLayerQGEqn&) = delete;
  TwoLayerQGEqn& operator=(const TwoLayerQGEqn&) = delete;
  void Solve(Field* psi1Prev, Field* omega1Prev, Field* psi2Prev, Field* omega2Prev) {
    se_ok(se_qg2_solve(h, psi1Prev ? psi1Prev->h : nullptr, omega1Prev ? omega1Prev->h : nullptr,
                       psi2Prev ? psi2Prev->h : nullptr, omega2Prev ? omega2Prev->h : nullptr));
  }
  se_qg2* h = nullptr;
};

/* BCs(bool* bottom, bool* top, bool* left, bool* right, mesh, 0), the
 * reference's per-component constructor (src/base/BCs.cpp:175-): one scalar
 * se_bcs per velocity component. */
class BCs2 {
 public:
  BCs2(bool* bottom, bool* top, bool* left, bool* right, Mesh* mesh) {
    se_ok(se_bcs_create(mesh->h, bottom[0], top[0], left[0], right[0], &u));
    se_ok(se_bcs_create(mesh->h, bottom[1], top[1], left[1], right[1], &v));
  }
  ~BCs2() {
    se_bcs_destroy(u);
    se_bcs_destroy(v);
  }
  BCs2(const BCs2&) = delete;
  BCs2& operator=(const BCs2&) = delete;
  se_bcs *u = nullptr, *v = nullptr;
};

/* NavierStokesEqn(velocity, pressure, dt, bcs) and Solve, src/ns/NavierStokesEqn.h. */
class NavierStokesEqn {
 public:
  NavierStokesEqn(Field* velocity, Field* pressure, double dt, BCs2* vbcs,
                  const char* options = "") {
    se_solver_opts o = se_options("helm_", options);
    se_ok(se_ns_create(velocity->h, pressure->h, vbcs ? vbcs->u : nullptr,
                       vbcs ? vbcs->v : nullptr, dt, &o, &h));
  }
  ~NavierStokesEqn() { se_ns_destroy(h); }
  NavierStokesEqn(const NavierStokesEqn&) = delete;
  NavierStokesEqn& operator=(const NavierStokesEqn&) = delete;
  void Solve(Field* velocity, Field* pressure, Field* prevVel, double nu, int svvCutoff) {
    se_ok(se_ns_solve(h, velocity->h, pressure->h, prevVel ? prevVel->h : nullptr, nu,
                      svvCutoff));
  }
  se_ns* h = nullptr;
};

#endif /* SEGPU_HPP */
