/* CPU restatement of SE's semi-Lagrangian + Helmholtz/Poisson hot path.
 *
 * TEST INFRASTRUCTURE ONLY: the oracle and the timed CPU baseline. Only
 * tests/, the smoke check and bench.py's CPU legs may load it; the product
 * (se_b200, include/segpu.h) never links or calls it.
 *
 * Parity status:
 *  - GLL tables, mesh, element search, interpolation, SL advection, element
 *    matrices, FieldRHS and the BCs maps restate src/base in the same
 *    operation order and are pinned bit-for-bit against the reference's own
 *    compiled code (oracle/_ref) and the fixtures in tests/golden/.
 *  - Global assembly, Dirichlet lifting, UpdateField, FieldError and the
 *    Jacobi-preconditioned CG restate code that needs PETSc (absent here):
 *    src/base/Matrix.cpp, Vector.cpp, Utils.cpp, src/linsys/HelmholtzEqn.cpp, PoissonEqn.cpp and PETSc's
 *    KSPCG/PCJACOBI semantics (third party, version unpinned). Their
 *    element-level inputs are pinned; the solver semantics are "parity
 *    unpinned" beyond that.
 */
#ifndef SE_ORACLE_H
#define SE_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

typedef struct or_mesh or_mesh;

/* GLL tables of order N (src/base/Legendre.cpp:15-95). */
void or_gll(int N, double* abcissa, double* weights, double* dCij, double* Pj);

or_mesh* or_mesh_create(int nx, int ny, int N, double x0, double y0, double x1,
                        double y1, int perx, int pery);
void or_mesh_destroy(or_mesh* m);
/* Test switch, not part of the reference: interpolate with extended-precision
 * Lagrange-product cardinal functions (same search, coordinates and snap). */
void or_mesh_set_accurate(or_mesh* m, int on);
int or_mesh_nverts(const or_mesh* m);
void or_mesh_verts(const or_mesh* m, double* out);
void or_global_to_local(const or_mesh* m, const double* pts, int npts, int* el,
                        double* lc);
void or_shape_funcs_at(const or_mesh* m, const double* coords, int npts, double* Ni);
void or_interp_global(const or_mesh* m, int ndofs, const double* vals,
                      const double* pts, int npts, double* out);
void or_interp_derivs_global(const or_mesh* m, const double* vals,
                             const double* pts, int npts, double* grad);

/* SL advection (src/base/Advector.cpp). field/vel are [Nv][ndofs] row-major;
 * field_prev == NULL selects first order. nthreads >= 1 splits the node loop.
 * Returns 0, or -1 for N < 3 (the bicubic path is not restated). */
int or_advect(const or_mesh* m, int ndofs, const double* field, const double* vel,
              const double* field_prev, const double* vel_prev, double dt,
              double* out, int nthreads);
/* First-order departure points and their elements. */
void or_departure_first(const or_mesh* m, const double* vel, double dt,
                        double* dep, int* el);
/* Second-order departure points x1, x2 and their elements. */
void or_departure_second(const or_mesh* m, const double* vel, const double* vel_prev,
                         double dt, double* x1, int* el1, double* x2, int* el2);

/* BCs maps (scalar field, src/base/BCs.cpp:14-195). Returns the number of
 * vector unknowns, or -1 for an unsupported configuration. */
int or_bcs_maps(const or_mesh* m, int bottom, int top, int left, int right,
                int* field_to_vec, int* vec_to_field);

/* Element matrix cMass*Mass + cLap*Laplacian (Operator.cpp:63-84,157-177).
 * quirk != 0 keeps the reference's detJac = 1 in the Laplacian. */
void or_element_matrix(const or_mesh* m, int el, double cMass, double cLap,
                       int quirk, double* M);
void or_field_rhs_element(const or_mesh* m, const double* vals, int el, double* rhs);

/* Assembled operator in CSR over the vector unknowns, plus the Dirichlet
 * lifting vector b = -A_{I,D} u_D taken from sol_vals. */
typedef struct {
  int n, nnz;
  int* rowptr;
  int* col;
  double* val;
  double* lift;
} or_csr;
or_csr* or_assemble(const or_mesh* m, const int* field_to_vec, int ng,
                    double cMass, double cLap, int quirk, const double* sol_vals);
/* The same with HelmholtzEqn's SVV operator (constant svvConstant, cutoff
 * svvCutoff; none when svvCutoff == 0) added to every element matrix. */
or_csr* or_assemble_svv(const or_mesh* m, const int* field_to_vec, int ng, double cMass,
                        double cLap, int quirk, const double* sol_vals, double svvConstant,
                        int svvCutoff);
/* SVV::AssembleElement (src/base/SVV.cpp:120-176): M += constant*(Lxx+Lyy).
 * Returns -1 if a dense inverse fails. */
int or_svv_element(const or_mesh* m, int el, double constant, int mN, double* M);
void or_csr_destroy(or_csr* A);
void or_csr_matvec(const or_csr* A, const double* x, double* y, int nthreads);
/* Vector::Assemble of FieldRHS(1.0) over rhs_vals into f[ng] (zeroed first). */
void or_assemble_rhs(const or_mesh* m, const int* field_to_vec, int ng,
                     const double* rhs_vals, double* f);

/* PETSc KSPCG + PCJACOBI restatement. norm_type: 0 preconditioned (PETSc
 * default), 1 unpreconditioned, 2 natural. Returns the KSP converged reason
 * code (2 RTOL, 3 ATOL, -3 ITS, -4 DTOL, -8 INDEFINITE_PC,
 * -9 NANORINF, -10 INDEFINITE_MAT). x is zeroed first. */
int or_pcg(const or_csr* A, const double* b, double* x, double rtol, double atol,
           double dtol, int max_it, int norm_type, int remove_null_space,
           int nthreads, int* its, double* rnorm, double* rnorm0);

/* Copy the vector back into the field and refresh periodic copies
 * (src/base/Vector.cpp:40-61). */
void or_update_field(const or_mesh* m, const int* vec_to_field, int ng,
                     const double* x, double* vals);
void or_periodic_update(const or_mesh* m, int ndofs, double* vals);

double or_integrate(const or_mesh* m, const double* vals);
/* FieldError (src/base/Utils.cpp:232-254): numeric vs analytic, both fields on m. */
double or_field_error(const or_mesh* m, const double* numeric, const double* analytic,
                      int normalise);
double or_calc_time_step(const or_mesh* m, const double* vel, double courant);

/* TwoLayerQGEqn pieces (src/qg/TwoLayerQGEqn.cpp): the assembled
 * DissipationRHS vector and the diagonal of the PV mass matrix, over the
 * unknowns of f2v. */
void or_dissipation_rhs(const or_mesh* m, const int* f2v, int ng, double constant,
                        const double* field, const double* tau, const double* omega_hat,
                        const double* tau_e, double rF, double Ei, double nu, double* f);
void or_mass_diag(const or_mesh* m, const int* f2v, int ng, double a, double* d);

#ifdef __cplusplus
}
#endif
#endif
