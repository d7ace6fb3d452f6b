/* segpu: B200-native semi-Lagrangian advection and spectral-element
 * Helmholtz/Poisson solves for SE (davelee2804/SE).
 *
 * C-ABI drop-in for SE's per-timestep hot path. Every object mirrors a
 * reference class; the comment above each entry point names the reference
 * interface it replaces (paths inside the SE checkout).
 *
 * Conventions
 *  - Every call returns an int status: SE_OK (0) or a negative SE_ERR_* code;
 *    se_last_error() gives a one-line message for the calling thread.
 *  - Host arrays are in the reference layout: a field of ndofs components on
 *    a mesh with nVertsTotal vertices is double[nVertsTotal][ndofs],
 *    row-major, vertex index = j*nVerts[0] + i (x fastest), periodic duplicate
 *    vertices stored (src/base/Field.cpp:17-35, src/base/Mesh.cpp:59-72).
 *  - Device state (field values, solver vectors) lives in GPU memory owned by
 *    the library; work is queued on the stream set by se_set_stream
 *    (default: the legacy default stream). Calls that return host results
 *    synchronise that stream.
 *  - Objects are not thread-safe; use one object per thread or serialise.
 *  - There is no CPU fallback: without a usable CUDA device every call that
 *    needs one fails with SE_ERR_CUDA.
 */
#ifndef SEGPU_H
#define SEGPU_H

#ifdef __cplusplus
extern "C" {
#endif

#define SE_OK 0
#define SE_ERR_ARG (-1)          /* invalid argument or handle */
#define SE_ERR_OOM (-2)          /* device or host allocation failed */
#define SE_ERR_CUDA (-3)         /* CUDA runtime error, or no CUDA device */
#define SE_ERR_UNSUPPORTED (-4)  /* configuration the reference supports but this build does not */
#define SE_ERR_NOT_CONVERGED (-5) /* solver stopped without converging; see se_solve_stats.reason */
#define SE_ERR_TIMEOUT (-6)      /* a bounded device-side wait gave up */
#define SE_ERR_DOMAIN (-7)       /* a departure point left the mesh after the periodic wrap */

/* PETSc-compatible converged reasons reported in se_solve_stats.reason. */
#define SE_KSP_CONVERGED_RTOL 2
#define SE_KSP_CONVERGED_ATOL 3
#define SE_KSP_DIVERGED_ITS (-3)
#define SE_KSP_DIVERGED_DTOL (-4)
#define SE_KSP_DIVERGED_BREAKDOWN (-5) /* FDM refinement stalled: no 10% gain in 3 steps */
#define SE_KSP_DIVERGED_INDEFINITE_PC (-8)
#define SE_KSP_DIVERGED_NANORINF (-9)
#define SE_KSP_DIVERGED_INDEFINITE_MAT (-10)

typedef struct se_mesh se_mesh;
typedef struct se_bcs se_bcs;
typedef struct se_field se_field;
typedef struct se_advector se_advector;
typedef struct se_linsys se_linsys; /* a HelmholtzEqn or a PoissonEqn */

/* Last error message of the calling thread ("" if none). */
const char* se_last_error(void);
/* Library version string. */
const char* se_version(void);
/* Stream for all subsequent device work of the calling process
 * (a cudaStream_t passed as void*; NULL = legacy default stream). */
int se_set_stream(void* stream);
/* Block until all queued device work of the library is done. */
int se_synchronize(void);

/* ------------------------------------------------------------------ Mesh --
 * Replaces Mesh::Mesh(name, nEls, "legendre", N, min, max, periodic)
 * (src/base/Mesh.h:6, src/base/Mesh.cpp:17-84). Only the GLL ("legendre")
 * element exists here; 2 <= N <= 12. */
int se_mesh_create(const int nEls[2], int N, const double min[2], const double max[2],
                   const int periodic[2], se_mesh** out);
int se_mesh_destroy(se_mesh* mesh);
/* nVerts[2], nVertsTotal (Mesh members, src/base/Mesh.h:11-13). */
int se_mesh_sizes(const se_mesh* mesh, int nVerts[2], int* nVertsTotal);
/* Mesh::verts as double[nVertsTotal][2] (src/base/Mesh.cpp:62-72). */
int se_mesh_verts(const se_mesh* mesh, double* verts);
/* GLL tables: abcissa[N+1], weights[N+1], dCij[(N+1)^2]
 * (src/base/Legendre.cpp:28-95). Any pointer may be NULL. */
int se_mesh_gll(const se_mesh* mesh, double* abcissa, double* weights, double* dCij);
/* Mesh::GlobalToLocal at npts host points (src/base/Mesh.cpp:109-176),
 * evaluated on the GPU: element index and local coordinates. */
int se_mesh_global_to_local(const se_mesh* mesh, const double* pts, int npts, int* el,
                            double* lcoord);

/* ------------------------------------------------------------------- BCs --
 * Replaces BCs::BCs(bottom, top, left, right, mesh, 0) for a scalar field
 * (src/base/BCs.h:3, src/base/BCs.cpp:36-195). */
int se_bcs_create(se_mesh* mesh, int bottom, int top, int left, int right, se_bcs** out);
int se_bcs_destroy(se_bcs* bcs);
/* Number of vector unknowns (nVertsTotal - size[0]). */
int se_bcs_vec_size(const se_bcs* bcs, int* n);
/* fieldToVecMap[nVertsTotal], vecToFieldMap[vec_size] (BCs members). */
int se_bcs_maps(const se_bcs* bcs, int* field_to_vec, int* vec_to_field);

/* ----------------------------------------------------------------- Field --
 * Replaces Field(name, mesh, nDofs, bcs) with its public double** vals
 * (src/base/Field.h:7-11). Values live on the GPU; upload/download move the
 * whole [nVertsTotal][ndofs] array. 1 <= ndofs <= 2. bcs may be NULL. */
int se_field_create(se_mesh* mesh, int ndofs, se_bcs* bcs, se_field** out);
int se_field_destroy(se_field* field);
int se_field_upload(se_field* field, const double* vals);
int se_field_download(const se_field* field, double* vals);
/* se_field_download queued on the library's stream without waiting (no
 * counterpart in the reference): vals must stay valid, and is complete after
 * se_synchronize or a wait on that stream; page-locked vals make the copy
 * overlap other streams' work. */
int se_field_download_async(const se_field* field, double* vals);
/* Device pointer to the values (double[nVertsTotal][ndofs]). */
int se_field_device_ptr(se_field* field, double** dptr);
/* Field::Copy (src/base/Field.cpp:49-55), device to device. */
int se_field_copy(se_field* dst, const se_field* src);
/* Field::PeriodicUpdate (src/base/Field.cpp:232-252). */
int se_field_periodic_update(se_field* field);
/* Field::Integrate(dof, average) (src/base/Field.cpp:181-200). */
int se_field_integrate(const se_field* field, int dof, int average, double* out);
/* Field::InterpGlobal at npts host points (src/base/Field.cpp:70-76);
 * out is double[npts][ndofs]. */
int se_field_interp_global(const se_field* field, const double* pts, int npts, double* out);

/* Field::Save(timeStep) / Field::Read(timeStep) (src/base/Field.cpp:256-368)
 * with a raw-binary file in place of HDF5: "<name>.<timeStep, 5 digits>.seb"
 * holds, in the HDF5 file's order, the magic "SEFIELD1", the dimensions
 * (int32, 2), the mesh resolution (int32 nVerts[0]-1, nVerts[1]-1), the rows
 * (int64 nVertsTotal) and columns (int32 nDofs), then the /data dataset as
 * double[rows][columns] in the reference's vertex order; little-endian.
 * Read checks the header against the field and fails with SE_ERR_ARG on a
 * mismatch, a missing or a truncated file. */
int se_field_save(const se_field* field, const char* name, int time_step);
int se_field_read(se_field* field, const char* name, int time_step);

/* Mesh::Save (src/base/Mesh.cpp:366-489) with a raw-binary file in place of
 * HDF5: "<name>.seb" holds, in the HDF5 file's order, the magic "SEMESH01",
 * the dimensions (int32 2, int32 0), the mesh resolution (int32 nVerts-1 per
 * direction), /min and /max (double[2] each), int64 nVertsTotal, int64 linear
 * quads, /vertices (double[nVertsTotal][2]) and /connectivity
 * (int32[quads][4], the reference's linear quads); little-endian, 72-byte
 * header. */
int se_mesh_save(const se_mesh* mesh, const char* name);

/* WriteXDMFHeader / WriteXDMF / WriteXDMFFooter / WriteXDMFTemporal
 * (src/base/Utils.cpp:53-229): the same files in the working directory
 * ("XDMF.<step>.xmf", "time.<step>.ts", "XDMF.temporalAll.xmf",
 * "XDMF.temporalFields.xmf", "XDMF.FilesField.xdmf") and the same grid,
 * topology, geometry and attribute structure, with Binary DataItems (byte
 * offset Seek, little-endian) into the mesh's and the fields' ".seb" files in
 * place of the HDF5 datasets. se_write_xdmf saves each field
 * (se_field_save(fields[i], names[i], time_step)); mesh_name names the file
 * se_mesh_save wrote. */
int se_write_xdmf_header(int time_step);
int se_write_xdmf(const se_field* const* fields, const char* const* names, int nfields,
                  const char* mesh_name, int time_step, double time, double dt);
int se_write_xdmf_footer(int time_step);
int se_write_xdmf_temporal(int n_time_steps, int dump_every);

/* TwoLayerQGEqn::GenVel / QuasiGeostrophicEqn::GenVel
 * (src/qg/TwoLayerQGEqn.cpp:335-352, src/qg/QuasiGeostrophicEqn.cpp:207-223):
 * vel (ndofs 2) = (-d psi/dy, d psi/dx) at every vertex, each derivative by
 * Field::InterpDerivsGlobal (src/base/Field.cpp:96-118) in the element that
 * Mesh::GetEl assigns to the vertex (at a shared vertex that element's
 * one-sided derivative, as in the reference). psi has ndofs 1, same mesh. */
int se_field_gen_vel(const se_field* psi, se_field* vel);

/* -------------------------------------------------------------- Advector --
 * Replaces Advector(field, velocity) (first order) and
 * Advector(field, velocity, fieldMinusOne, velMinusOne) (second order),
 * Advect(dt) and the public fieldSL (src/base/Advector.h:3-15,
 * src/base/Advector.cpp:51-246). velocity fields have ndofs = 2 and share the
 * field's mesh. N >= 3 (the reference's bicubic path for N < 3 is not built).
 * The advector keeps pointers to the fields; they must outlive it. */
int se_advector_create(se_field* field, se_field* velocity, se_field* field_prev,
                       se_field* vel_prev, se_advector** out);
int se_advector_destroy(se_advector* adv);
/* Advector::Advect(dt): writes fieldSL. */
int se_advect(se_advector* adv, double dt);
/* The advector's fieldSL (owned by the advector). */
int se_advector_field_sl(se_advector* adv, se_field** field_sl);
/* Departure data of the last se_advect: element index of every vertex's
 * departure point (second order: x1 then x2), as Mesh::GetEl assigns them.
 * el has nVertsTotal (first order) or 2*nVertsTotal (second order) entries;
 * xy (nullable) gets the coordinates. Enables recording on the first call. */
int se_advector_departures(se_advector* adv, int* el, double* xy);

/* ----------------------------------------------------------- linear solve --
 * Solver options: SE's KSP options database entries
 * (-<prefix>ksp_type cg -<prefix>pc_type jacobi -<prefix>ksp_rtol ...). */
#define SE_NORM_PRECONDITIONED 0
#define SE_NORM_UNPRECONDITIONED 1
#define SE_NORM_NATURAL 2
#define SE_MODE_REFERENCE 0 /* the reference's Laplacian with detJac forced to 1 (src/base/Operator.cpp:72) */
#define SE_MODE_EXACT 1     /* the Laplacian with its true Jacobian */
#define SE_PREC_FP64 0      /* every operation in FP64: the drop-in */
#define SE_PREC_MIXED 1     /* FDM only: every refinement step's inverse on the tcgen05 tensor
                               cores (TF32 hi/lo operand pairs, FP32 accumulation, about 1e-6
                               relative); residuals, norms and the solution in FP64 */
#define SE_PREC_BF16 2      /* SE_METHOD_CG: FP64 iterative refinement around a CG whose
                               operator apply reads its direction vector in BF16 and computes
                               in FP32 (dots, updates, residuals FP64; orders 4-8, no SVV, no
                               null-space removal). SE_METHOD_FDM: BF16 data,
                               FP32-accumulated inner inverses, FP64 refinement; converges only
                               while 2^-8 times the operator's condition number stays below 1
                               and otherwise stops with SE_KSP_DIVERGED_BREAKDOWN */
#define SE_PREC_FP16 3      /* SE_METHOD_CG: as SE_PREC_BF16 with an FP16 direction vector
                               (each inner solve scaled into FP16's range); also the FP16
                               input of se_linsys_apply_low */
#define SE_PREC_FP64_TC 4   /* FDM only: the first refinement step's inverse in FP64, the
                               following ones as SE_PREC_MIXED */
#define SE_METHOD_CG 0      /* PETSc KSPCG + PCJACOBI semantics: the drop-in (FP64; BF16/FP16 as above) */
#define SE_METHOD_FDM 1     /* fast diagonalization: exact inverse by 1-D eigenvector transforms */
typedef struct {
  double rtol;    /* default 1e-5 (PETSc) */
  double atol;    /* default 1e-50 */
  double dtol;    /* default 1e5 */
  int max_it;     /* default 10000 */
  int norm_type;  /* SE_NORM_*, default preconditioned */
  int mode;       /* SE_MODE_*, default SE_MODE_REFERENCE */
  int precision;  /* SE_PREC_*, default SE_PREC_FP64 */
  int inner_max_it; /* reserved (default 2000) */
  double inner_rtol; /* reserved (default 1e-6) */
  int method;     /* SE_METHOD_*, default SE_METHOD_CG. FDM: the solution of
                     A x = b by fast diagonalization, refined in FP64 until the
                     chosen residual norm meets rtol/atol (its = refinement
                     steps); precision selects the GEMM arithmetic. */
} se_solver_opts;

typedef struct {
  int reason;     /* SE_KSP_* */
  int its;        /* CG iterations (mixed: inner iterations summed) */
  int outer_its;  /* mixed: refinement steps; FP64: 0 */
  double rnorm;   /* final residual norm in the chosen norm */
  double rnorm0;  /* initial residual norm in the chosen norm */
  double kernel_ms; /* device time of the CG launch(es), CUDA events */
} se_solve_stats;

int se_solver_opts_default(se_solver_opts* opts);
/* Parse a PETSc-style options string for one prefix, e.g.
 * "-helm_ksp_rtol 1e-10 -helm_ksp_max_it 500", into opts. Unknown options
 * and other prefixes are ignored; a ksp_type other than cg or preonly, or a
 * pc_type other than jacobi or fdm, returns SE_ERR_UNSUPPORTED. One key is
 * this library's own: -<prefix>precision fp64|mixed|fp64_tc|bf16|fp16 sets
 * opts->precision. */
int se_solver_opts_parse(se_solver_opts* opts, const char* prefix, const char* options);

/* Replaces HelmholtzEqn(sol, rhs, c, nu, dt, svvCutoff)
 * (src/linsys/HelmholtzEqn.h:3, src/linsys/HelmholtzEqn.cpp:43-104):
 * A = c*Mass + nu*dt*Laplacian on sol's mesh and boundary conditions, plus
 * with 0 < svvCutoff <= N the spectral vanishing viscosity operator
 * SVV(dt, svvCutoff) (src/base/SVV.cpp:50-176) as the reference builds it
 * (its y term formed from the x derivative, as the reference forms it; the
 * true Jacobian in either mode). rhs may be NULL (right-hand side = Dirichlet
 * lifting only). An SVV system is solved by CG (SE_METHOD_FDM, the FDM
 * inverse and the low-precision apply return SE_ERR_UNSUPPORTED for it). */
int se_helmholtz_create(se_field* sol, se_field* rhs, double c, double nu, double dt,
                        int svvCutoff, const se_solver_opts* opts, se_linsys** out);
/* Replaces PoissonEqn(sol, rhs, c) (src/linsys/PoissonEqn.cpp:30-80):
 * A = c*Laplacian. */
int se_poisson_create(se_field* sol, se_field* rhs, double c, const se_solver_opts* opts,
                      se_linsys** out);
int se_linsys_destroy(se_linsys* ls);
int se_linsys_set_opts(se_linsys* ls, const se_solver_opts* opts);
/* HelmholtzEqn::Assemble / PoissonEqn::Assemble
 * (src/linsys/HelmholtzEqn.cpp:113-125): captures the Dirichlet lifting
 * from the current boundary values of sol. Called by the first solve if not
 * called before. */
int se_linsys_assemble(se_linsys* ls);
/* HelmholtzEqn::Solve(name, removeNullSpace) / PoissonEqn::Solve
 * (src/linsys/HelmholtzEqn.cpp:127-158, src/linsys/PoissonEqn.cpp:102-134):
 * f = Mass*rhs + lifting, CG + Jacobi with zero initial guess, solution
 * copied into sol's unknowns and periodic copies. stats may be NULL.
 * remove_null_space: 0 none; 1 the constant null space projected out of
 * every preconditioned residual, as PETSc does (a right-hand side off the
 * operator's range then stagnates and ends with
 * SE_KSP_DIVERGED_INDEFINITE_PC, as in the reference); 2 the same after
 * replacing f by f - (sum f / sum d) d, d the operator diagonal: the
 * consistent system that iteration approaches, which converges (no
 * counterpart in the reference). The FDM method always solves that
 * consistent system when the null space is removed.
 * Returns SE_ERR_NOT_CONVERGED if the reason is negative. */
int se_linsys_solve(se_linsys* ls, int remove_null_space, se_solve_stats* stats);
/* Several solves in one call (the batched ensemble; no counterpart in the
 * reference, which solves one system at a time through the same Solve).
 * Systems using SE_METHOD_CG and the same polynomial order run as one
 * persistent cooperative launch (up to 256 per launch) whose launch shape is
 * chosen by a built-in autotuner on the first batch of a given signature;
 * SE_METHOD_FDM systems run their solve graphs overlapped on a pool of 8
 * streams. stats (nullable) gets one entry per system; the return value is
 * SE_ERR_NOT_CONVERGED if any system diverged. The caller's stream is ordered
 * after all solves. */
int se_linsys_solve_batch(se_linsys** systems, int n, int remove_null_space,
                          se_solve_stats* stats);
/* Queue a solve on the calling thread's stream without waiting (no
 * counterpart in the reference; for callers that overlap solves with other
 * work, such as the serving loop). SE_METHOD_FDM solves are fully
 * asynchronous; SE_METHOD_CG solves run to completion inside this call.
 * Exactly one se_linsys_solve_finish must follow: it waits for the solve,
 * fills stats (nullable) and returns what se_linsys_solve would have. */
int se_linsys_solve_async(se_linsys* ls, int remove_null_space);
int se_linsys_solve_finish(se_linsys* ls, se_solve_stats* stats);
/* y = A x on vector unknowns (device pointers, vec_size entries each), on
 * the calling thread's stream. Orders 4 to 8 return once the apply is
 * queued; orders 2, 3 and 9 to 12 (a TMA-staged kernel with bounded waits)
 * return after it has finished, with SE_ERR_TIMEOUT if a stage never
 * arrived. */
int se_linsys_apply(se_linsys* ls, const double* x_dev, double* y_dev);
/* No counterpart in the reference: x = A^{-1} r by the fast-diagonalization
 * transforms in FP64 (four tensor-core products; exact up to rounding, the
 * null mode of a singular operator set to zero), on the calling thread's
 * stream; device pointers, vec_size entries each, not aliased. A
 * preconditioner for callers that run their own Krylov loop. The first call
 * on a system computes its 1-D eigendecompositions (host work, allocation). */
int se_linsys_fdm_apply(se_linsys* ls, const double* r_dev, double* x_dev);
/* No counterpart in the reference: r = b - A x with the operator's sums and
 * the subtraction in double-double (rounded once), the residual of the
 * FP64 iterative refinement, for callers that refine themselves; device
 * pointers, vec_size entries each, r not aliasing x or b; queued on the
 * calling thread's stream. */
int se_linsys_residual(se_linsys* ls, const double* x_dev, const double* b_dev, double* r_dev);
/* No counterpart in the reference: x = A^{-1} r by the fast-diagonalization
 * transforms in FP64 (precision SE_PREC_FP64, as se_linsys_fdm_apply) or on
 * the tcgen05 tensor cores (SE_PREC_MIXED: r split into TF32 hi/lo pairs,
 * three TF32 products per K step with FP32 accumulation, about 1e-6
 * relative), the inner solve of the mixed-precision refinement; same
 * arguments and rules as se_linsys_fdm_apply. */
int se_linsys_fdm_apply_prec(se_linsys* ls, int precision, const double* r_dev, double* x_dev);
/* No counterpart in the reference: y = A x with x in BF16 or FP16
 * (precision SE_PREC_BF16 / SE_PREC_FP16) and y in FP32, the operator and
 * the arithmetic in FP32 (device pointers, vec_size entries each). */
int se_linsys_apply_low(se_linsys* ls, int precision, const void* x_dev, float* y_dev);
/* The Jacobi diagonal of A (device pointer, vec_size entries). */
int se_linsys_diagonal(se_linsys* ls, double* d_dev);
int se_linsys_vec_size(const se_linsys* ls, int* n);

/* No counterpart in the reference: HelmholtzEqn/PoissonEqn construction,
 * Assemble and Solve in one call that allocates no memory, for callers that
 * cannot call cudaMalloc (a driver that reserves its whole device-memory
 * budget at start-up while other components share the GPU, or a time loop
 * that cannot take the device-wide synchronisation cudaMalloc/cudaFree may
 * cause mid-step). The mesh is given by the Mesh/BCs constructor arguments
 * (bcs = {bottom, top, left, right}); rhs_dev (nullable) and sol_dev are
 * caller-owned device arrays of nVertsTotal doubles in the reference's vertex
 * order; sol_dev holds the Dirichlet values on entry and the solution on
 * return. poisson != 0 selects A = c*Laplacian (nu, dt ignored). It runs
 * the drop-in solver only (Jacobi CG in FP64, PETSc KSPCG semantics): options
 * are checked as se_helmholtz_create checks them, and method != SE_METHOD_CG
 * or precision != SE_PREC_FP64 returns SE_ERR_UNSUPPORTED.
 * Limit: at most 65536 vector unknowns (e.g. 32x32 elements at N = 8);
 * larger systems return SE_ERR_UNSUPPORTED. All temporaries live in one
 * static device array of about 5 MB that every GPU loading the library
 * holds until exit; every call shares it and leaves its contents behind.
 * Two calls whose device work overlapped would race on it, so the library
 * serialises them: each call holds a process-wide lock until its device work
 * has finished (it returns after a stream synchronize). The first call on a
 * device looks the array up (cudaGetSymbolAddress) and should come before
 * any stream capture. */
int se_helmholtz_solve_noalloc(const int nEls[2], int N, const double min[2],
                               const double max[2], const int periodic[2], const int bcs[4],
                               double c, double nu, double dt, int poisson,
                               const se_solver_opts* opts, int remove_null_space,
                               const double* rhs_dev, double* sol_dev, se_solve_stats* stats);

/* ---------------------------------------------------------------- serving --
 * A continuous-batching request server (no counterpart in the reference,
 * which runs one model in one process). A worker thread admits queued
 * requests in arrival order into free execution slots (one CUDA stream each)
 * whenever the device-memory budget allows their resources, queues each
 * request's device work without waiting, and completes requests as their
 * streams finish, so requests that arrive while others run overlap on the
 * device. Resources are cached per configuration and reused; least recently
 * used idle ones are released when a new configuration needs the memory.
 * Results do not depend on what else runs: the kernels are deterministic. */
#define SE_REQ_HELMHOLTZ 0 /* one HelmholtzEqn/PoissonEqn solve */
#define SE_REQ_ADVECT 1    /* steps of first-order SL advection of a tracer */
typedef struct {
  int kind;                 /* SE_REQ_* */
  int nEls[2];              /* mesh, as se_mesh_create */
  int N;
  double min[2], max[2];
  int periodic[2];
  int bcs[4];               /* Helmholtz: Dirichlet bottom, top, left, right */
  double c, nu, dt;         /* Helmholtz: A = c*Mass + nu*dt*Laplacian */
  int poisson;              /* Helmholtz: nonzero for A = c*Laplacian */
  se_solver_opts opts;      /* Helmholtz: solver options */
  int steps;                /* advection: number of steps */
  double sl_dt;             /* advection: time step */
  const double* in;         /* host [nVertsTotal]: right-hand side field / tracer */
  const double* aux;        /* host: solution field with its Dirichlet values [nVertsTotal]
                               (NULL: zeros) / velocity [nVertsTotal][2] */
  double* out;              /* host [nVertsTotal]: solution / advected tracer */
} se_request;                /* host buffers must stay valid until se_server_wait returns;
                               page-locked ones (cudaMallocHost / cudaHostRegister) are
                               copied directly, others through the server's staging */
typedef struct {
  int status;               /* SE_OK or SE_ERR_* */
  int reason, its;          /* Helmholtz: solver reason and iterations */
  double queued_ms;         /* submission to admission */
  double latency_ms;        /* submission to result in out */
  char error[160];          /* status != SE_OK: the failing call's message */
} se_result;
typedef struct se_server se_server;
/* slots: concurrent requests (1..64); device_gib: memory budget for cached
 * request resources. Work runs on the device current at creation. */
int se_server_create(int slots, double device_gib, se_server** out);
int se_server_submit(se_server* srv, const se_request* req, long long* ticket);
/* Wait for a request; res (nullable) gets its status and timings. */
int se_server_wait(se_server* srv, long long ticket, se_result* res);
/* Finish queued work, then release everything. */
int se_server_destroy(se_server* srv);

/* ------------------------------------------------------------ utilities -- */
/* ------------------------------------------------------ two-layer QG step --
 * Replaces TwoLayerQGEqn(psi1, omega1, psi2, omega2, F1, F2, beta, E2, r, nu,
 * tau_e, dt) and its Solve (src/qg/TwoLayerQGEqn.h, .cpp:17-433): one step of
 * the two-layer quasi-geostrophic model, on the device: PV of both layers
 * (GenPV), SL advection of PV by the GenVel velocities (first order, or
 * second order when the previous fields are given), baroclinic Helmholtz
 * (c = -(F1+F2)) and barotropic Poisson (c = -1) inversions with the given
 * solver options, the dissipative PV update (SolveQ with DissipationRHS),
 * the second inversions and the update of psi1, psi2, omega1, omega2 in
 * place. The reference's own step is kept as it is: the first-order step
 * applies SolveQ to layer 1 only, both layers' dissipation uses the first
 * baroclinic solution, and the PV mass matrix is scaled by 1.5 from the first
 * second-order step on. Scalar fields on one mesh; psi1's boundary conditions
 * (e.g. walls in y of a channel) are those of the inversions; tau_e is the
 * radiative-equilibrium field of the dissipation. The fields must outlive the
 * object. */
typedef struct se_qg2 se_qg2;
int se_qg2_create(se_field* psi1, se_field* omega1, se_field* psi2, se_field* omega2, double F1,
                  double F2, double beta, double E2, double r, double nu, se_field* tau_e,
                  double dt, const se_solver_opts* opts, se_qg2** out);
/* TwoLayerQGEqn::Solve(psi1Prev, omega1Prev, psi2Prev, omega2Prev): second
 * order when all four previous fields are given (they are then replaced by
 * the fields as they were before this step), first order when all are NULL.
 * A solve that does not converge leaves its last iterate and the step goes
 * on (the reference never checks); the call then returns
 * SE_ERR_NOT_CONVERGED with the step complete. */
int se_qg2_solve(se_qg2* qg, se_field* psi1_prev, se_field* omega1_prev, se_field* psi2_prev,
                 se_field* omega2_prev);
int se_qg2_destroy(se_qg2* qg);

/* ------------------------------------------- Navier-Stokes splitting step --
 * Replaces NavierStokesEqn(velocity, pressure, dt) and its Solve
 * (src/ns/NavierStokesEqn.h, .cpp:23-147): one step of the incompressible
 * splitting scheme on the device: SL advection of the velocity by itself
 * (first order, or second order with the previous velocity), the divergence
 * of the advected velocity at every vertex (times 1.5 times 10.0 in the
 * second-order step, as the reference writes it), the pressure Poisson solve
 * (c = -dt, constant null space removed), the pressure-gradient correction
 * and the viscous Helmholtz solve (c = 1.0, then 1.5 from the first
 * second-order step on; nu and dt) into the velocity in place.
 * velocity has 2 components; pressure 1 component on a mesh of the same
 * geometry (the same object or the same parameters). The reference's
 * per-component velocity BCs (BCs(bool*, bool*, bool*, bool*),
 * src/base/BCs.cpp:175-) are given as one scalar se_bcs per component on the
 * velocity's mesh (NULL: no Dirichlet sides); the velocity's own bcs are not
 * used. The component systems are block-diagonal in the reference's
 * interleaved matrix (src/base/Operator.cpp:67-79, :161-172) and are solved
 * as two scalar systems. The fields must outlive the object. */
typedef struct se_ns se_ns;
int se_ns_create(se_field* velocity, se_field* pressure, se_bcs* bcs_u, se_bcs* bcs_v, double dt,
                 const se_solver_opts* opts, se_ns** out);
/* NavierStokesEqn::Solve(velocity, pressure, prevVel, nu, svvCutoff):
 * velocity and pressure must be the fields the object was made with; prevVel
 * NULL for the first-order step (it is read, not changed); nu and svvCutoff
 * (0 <= svvCutoff <= N) are taken when the viscous systems are made (first
 * call of each order), as in the reference; with svvCutoff != 0 those
 * systems carry the SVV operator and are solved by CG whatever the options'
 * method (no fast diagonalization holds for them). A solve that does not converge leaves
 * its last iterate and the step goes on, as in the reference; the call then
 * returns SE_ERR_NOT_CONVERGED with the step complete (se_ns_stats shows
 * which). */
int se_ns_solve(se_ns* ns, se_field* velocity, se_field* pressure, se_field* prev_vel, double nu,
                int svvCutoff);
/* Solver statistics of the last step: [0] pressure, [1] u, [2] v. */
int se_ns_stats(const se_ns* ns, se_solve_stats stats[3]);
int se_ns_destroy(se_ns* ns);

/* CalcTimeStep(velocity, courantNo) (src/base/Utils.cpp:23-40). */
int se_calc_time_step(const se_field* velocity, double courant, double* dt);
/* FieldError(numeric, analytic, dof, normalise) (src/base/Utils.cpp:232-254). */
int se_field_error(const se_field* numeric, const se_field* analytic, int dof, int normalise,
                   double* err);

#ifdef __cplusplus
}
#endif
#endif /* SEGPU_H */
