"""ctypes bindings to the CPU oracle. TEST INFRASTRUCTURE ONLY.

Two libraries, both built by ``oracle/Makefile``:

* ``oracle/_build/libseoracle.so`` -- the C restatement (``se_oracle.c``) of
  SE's semi-Lagrangian + Helmholtz/Poisson path, the oracle proper and the
  timed CPU baseline.
* ``oracle/_ref/libseref.so`` -- the reference's own ``src/base`` sources
  compiled unmodified behind ``ref_shim.cpp``; used to pin the restatement.
  It is built only where the reference checkout exists and travels as a
  prebuilt file; callers must tolerate its absence (``ref_available()``).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU legs import
this module, and only as the checker or the CPU baseline.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "libseoracle.so")
REF_SO = os.path.join(HERE, "_ref", "libseref.so")
# the reference checkout (its src/base is compiled into _ref/ when given)
REF_SRC = os.environ.get("SE_REFERENCE_SRC", "")

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)
_dbl = ctypes.c_double
_int = ctypes.c_int
_vp = ctypes.c_void_p


def build(with_ref: bool | None = None) -> None:
    """Compile the restatement, and the reference library when its sources exist."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    if with_ref is None:
        with_ref = bool(REF_SRC) and os.path.isdir(os.path.join(REF_SRC, "src", "base"))
    if with_ref:
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={REF_SRC}"], check=True)


def _pd(a):
    return None if a is None else a.ctypes.data_as(_D)


def _pi(a):
    return None if a is None else a.ctypes.data_as(_I)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build(with_ref=False)
        L = ctypes.CDLL(ORACLE_SO)
        L.or_mesh_create.restype = _vp
        L.or_mesh_create.argtypes = [_int, _int, _int, _dbl, _dbl, _dbl, _dbl, _int, _int]
        L.or_mesh_destroy.argtypes = [_vp]
        L.or_mesh_set_accurate.argtypes = [_vp, _int]
        L.or_mesh_nverts.argtypes = [_vp]
        L.or_mesh_verts.argtypes = [_vp, _D]
        L.or_gll.argtypes = [_int, _D, _D, _D, _D]
        L.or_global_to_local.argtypes = [_vp, _D, _int, _I, _D]
        L.or_shape_funcs_at.argtypes = [_vp, _D, _int, _D]
        L.or_interp_global.argtypes = [_vp, _int, _D, _D, _int, _D]
        L.or_interp_derivs_global.argtypes = [_vp, _D, _D, _int, _D]
        L.or_advect.argtypes = [_vp, _int, _D, _D, _D, _D, _dbl, _D, _int]
        L.or_departure_first.argtypes = [_vp, _D, _dbl, _D, _I]
        L.or_departure_second.argtypes = [_vp, _D, _D, _dbl, _D, _I, _D, _I]
        L.or_bcs_maps.argtypes = [_vp, _int, _int, _int, _int, _I, _I]
        L.or_element_matrix.argtypes = [_vp, _int, _dbl, _dbl, _int, _D]
        L.or_field_rhs_element.argtypes = [_vp, _D, _int, _D]
        L.or_assemble.restype = _vp
        L.or_assemble.argtypes = [_vp, _I, _int, _dbl, _dbl, _int, _D]
        L.or_assemble_svv.restype = _vp
        L.or_assemble_svv.argtypes = [_vp, _I, _int, _dbl, _dbl, _int, _D, _dbl, _int]
        L.or_svv_element.argtypes = [_vp, _int, _dbl, _int, _D]
        L.or_csr_destroy.argtypes = [_vp]
        L.or_csr_matvec.argtypes = [_vp, _D, _D, _int]
        L.or_assemble_rhs.argtypes = [_vp, _I, _int, _D, _D]
        L.or_pcg.argtypes = [_vp, _D, _D, _dbl, _dbl, _dbl, _int, _int, _int, _int,
                             _I, _D, _D]
        L.or_update_field.argtypes = [_vp, _I, _int, _D, _D]
        L.or_periodic_update.argtypes = [_vp, _int, _D]
        L.or_integrate.restype = _dbl
        L.or_integrate.argtypes = [_vp, _D]
        L.or_field_error.restype = _dbl
        L.or_field_error.argtypes = [_vp, _D, _D, _int]
        L.or_calc_time_step.restype = _dbl
        L.or_calc_time_step.argtypes = [_vp, _D, _dbl]
        L.or_dissipation_rhs.argtypes = [_vp, _I, _int, _dbl, _D, _D, _D, _D, _dbl, _dbl, _dbl,
                                         _D]
        L.or_mass_diag.argtypes = [_vp, _I, _int, _dbl, _D]
        _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref():
    """The reference's own compiled src/base (raises if it was never built)."""
    global _ref
    if _ref is None:
        if not os.path.exists(REF_SO):
            raise FileNotFoundError(REF_SO)
        R = ctypes.CDLL(REF_SO)
        R.ref_gll.argtypes = [_int, _D, _D, _D, _D]
        R.ref_shape_funcs_at.argtypes = [_int, _D, _int, _D]
        R.ref_mesh_create.restype = _vp
        R.ref_mesh_create.argtypes = [_int, _int, _int, _dbl, _dbl, _dbl, _dbl, _int, _int]
        R.ref_mesh_destroy.argtypes = [_vp]
        R.ref_mesh_nverts.argtypes = [_vp]
        R.ref_mesh_verts.argtypes = [_vp, _D]
        R.ref_global_to_local.argtypes = [_vp, _D, _int, _I, _D]
        R.ref_bcs_create.restype = _vp
        R.ref_bcs_create.argtypes = [_vp, _int, _int, _int, _int]
        R.ref_bcs_destroy.argtypes = [_vp]
        R.ref_bcs_vecsize.argtypes = [_vp]
        R.ref_bcs_maps.argtypes = [_vp, _I, _I]
        R.ref_element_matrix.argtypes = [_vp, _int, _dbl, _dbl, _D]
        R.ref_svv_element.argtypes = [_vp, _int, _dbl, _int, _D]
        R.ref_field_rhs_element.argtypes = [_vp, _D, _int, _D]
        R.ref_advect.argtypes = [_vp, _int, _D, _D, _D, _D, _dbl, _D]
        R.ref_departure_first.argtypes = [_vp, _D, _dbl, _D, _I]
        R.ref_interp_derivs_global.argtypes = [_vp, _D, _D, _int, _D]
        R.ref_interp_global.argtypes = [_vp, _int, _D, _D, _int, _D]
        R.ref_integrate.restype = _dbl
        R.ref_integrate.argtypes = [_vp, _D]
        _ref = R
    return _ref


def gll(N: int, use_ref: bool = False):
    a, w, pj = np.zeros(N + 1), np.zeros(N + 1), np.zeros(N + 1)
    dc = np.zeros((N + 1) * (N + 1))
    (ref().ref_gll if use_ref else lib().or_gll)(N, _pd(a), _pd(w), _pd(dc), _pd(pj))
    return a, w, dc.reshape(N + 1, N + 1), pj


class Mesh:
    """A reference-layout mesh held by the restatement (``use_ref=False``) or
    by the reference's own ``Mesh`` class (``use_ref=True``)."""

    def __init__(self, nx, ny, N, lo=(0.0, 0.0), hi=(1.0, 1.0), periodic=(True, True),
                 use_ref=False, accurate=False):
        self.nx, self.ny, self.N = nx, ny, N
        self.lo, self.hi, self.periodic = tuple(lo), tuple(hi), tuple(bool(p) for p in periodic)
        self.use_ref = use_ref
        self.L = ref() if use_ref else lib()
        create = self.L.ref_mesh_create if use_ref else self.L.or_mesh_create
        self.h = create(nx, ny, N, lo[0], lo[1], hi[0], hi[1], int(periodic[0]), int(periodic[1]))
        if not self.h:
            raise ValueError("mesh rejected")
        if accurate:
            assert not use_ref, "the reference has only its own formula"
            self.L.or_mesh_set_accurate(self.h, 1)
        self.nvx, self.nvy = nx * N + 1, ny * N + 1
        self.nv = self.nvx * self.nvy

    def close(self):
        if self.h:
            (self.L.ref_mesh_destroy if self.use_ref else self.L.or_mesh_destroy)(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _fn(self, name):
        return getattr(self.L, ("ref_" if self.use_ref else "or_") + name)

    def verts(self):
        v = np.zeros((self.nv, 2))
        self._fn("mesh_verts")(self.h, _pd(v))
        return v

    def global_to_local(self, pts):
        pts = _f64(pts).reshape(-1, 2)
        el = np.zeros(len(pts), dtype=np.int32)
        lc = np.zeros_like(pts)
        self._fn("global_to_local")(self.h, _pd(pts), len(pts), _pi(el), _pd(lc))
        return el, lc

    def interp_global(self, vals, pts, ndofs=1):
        vals, pts = _f64(vals), _f64(pts).reshape(-1, 2)
        out = np.zeros((len(pts), ndofs))
        self._fn("interp_global")(self.h, ndofs, _pd(vals), _pd(pts), len(pts), _pd(out))
        return out

    def interp_derivs_global(self, vals, pts):
        vals, pts = _f64(vals), _f64(pts).reshape(-1, 2)
        out = np.zeros((len(pts), 2))
        self._fn("interp_derivs_global")(self.h, _pd(vals), _pd(pts), len(pts), _pd(out))
        return out

    def advect(self, field, vel, dt, field_prev=None, vel_prev=None, nthreads=1):
        field = _f64(field)
        ndofs = 1 if field.ndim == 1 else field.shape[1]
        vel = _f64(vel)
        fp = None if field_prev is None else _f64(field_prev)
        vp = None if vel_prev is None else _f64(vel_prev)
        out = np.zeros_like(field)
        if self.use_ref:
            self.L.ref_advect(self.h, ndofs, _pd(field), _pd(vel), _pd(fp), _pd(vp), dt, _pd(out))
        else:
            rc = self.L.or_advect(self.h, ndofs, _pd(field), _pd(vel), _pd(fp), _pd(vp), dt,
                                  _pd(out), nthreads)
            if rc != 0:
                raise ValueError("SL advection needs N >= 3")
        return out

    def departure_first(self, vel, dt):
        vel = _f64(vel)
        dep = np.zeros((self.nv, 2))
        el = np.zeros(self.nv, dtype=np.int32)
        self._fn("departure_first")(self.h, _pd(vel), dt, _pd(dep), _pi(el))
        return dep, el

    def departure_second(self, vel, vel_prev, dt):
        assert not self.use_ref
        vel, vel_prev = _f64(vel), _f64(vel_prev)
        x1, x2 = np.zeros((self.nv, 2)), np.zeros((self.nv, 2))
        e1, e2 = np.zeros(self.nv, dtype=np.int32), np.zeros(self.nv, dtype=np.int32)
        self.L.or_departure_second(self.h, _pd(vel), _pd(vel_prev), dt, _pd(x1), _pi(e1),
                                   _pd(x2), _pi(e2))
        return x1, e1, x2, e2

    def element_matrix(self, el, c_mass, c_lap, quirk=True):
        nn = (self.N + 1) ** 2
        M = np.zeros(nn * nn)
        if self.use_ref:
            assert quirk, "the reference only has its own Laplacian"
            self.L.ref_element_matrix(self.h, el, c_mass, c_lap, _pd(M))
        else:
            self.L.or_element_matrix(self.h, el, c_mass, c_lap, int(bool(quirk)), _pd(M))
        return M.reshape(nn, nn)

    def svv_element(self, el, constant, cutoff):
        """SVV(constant, cutoff)'s element matrix (SVV::AssembleElement)."""
        nn = (self.N + 1) ** 2
        M = np.zeros(nn * nn)
        if self.use_ref:
            self.L.ref_svv_element(self.h, el, constant, cutoff, _pd(M))
        elif self.L.or_svv_element(self.h, el, constant, cutoff, _pd(M)) != 0:
            raise ValueError("singular dense matrix in the SVV element")
        return M.reshape(nn, nn)

    def field_rhs_element(self, vals, el):
        vals = _f64(vals)
        out = np.zeros((self.N + 1) ** 2)
        self._fn("field_rhs_element")(self.h, _pd(vals), el, _pd(out))
        return out

    def bcs_maps(self, bottom=False, top=False, left=False, right=False):
        f2v = np.zeros(self.nv, dtype=np.int32)
        if self.use_ref:
            b = self.L.ref_bcs_create(self.h, int(bottom), int(top), int(left), int(right))
            ng = self.L.ref_bcs_vecsize(b)
            v2f = np.zeros(ng, dtype=np.int32)
            self.L.ref_bcs_maps(b, _pi(f2v), _pi(v2f))
            self.L.ref_bcs_destroy(b)
            return f2v, v2f
        v2f = np.zeros(self.nv, dtype=np.int32)
        ng = self.L.or_bcs_maps(self.h, int(bottom), int(top), int(left), int(right),
                                _pi(f2v), _pi(v2f))
        if ng < 0:
            raise ValueError("unsupported boundary configuration")
        return f2v, v2f[:ng].copy()

    def integrate(self, vals):
        return self._fn("integrate")(self.h, _pd(_f64(vals)))

    # -- restatement only ------------------------------------------------
    def field_error(self, numeric, analytic, normalise=True):
        return self.L.or_field_error(self.h, _pd(_f64(numeric)), _pd(_f64(analytic)),
                                     int(normalise))

    def calc_time_step(self, vel, courant):
        return self.L.or_calc_time_step(self.h, _pd(_f64(vel)), courant)

    def periodic_update(self, vals, ndofs=1):
        vals = _f64(vals).copy()
        self.L.or_periodic_update(self.h, ndofs, _pd(vals))
        return vals


class CSR:
    """The assembled operator (or_assemble): c_mass*Mass + c_lap*Laplacian,
    plus SVV(constant, cutoff) when svv = (constant, cutoff) is given."""

    def __init__(self, mesh: Mesh, f2v, ng, c_mass, c_lap, quirk=True, sol_vals=None, svv=None):
        assert not mesh.use_ref
        self.mesh, self.L = mesh, mesh.L
        self.f2v = np.ascontiguousarray(f2v, dtype=np.int32)
        sv = None if sol_vals is None else _f64(sol_vals)
        svc, svn = (0.0, 0) if svv is None else (float(svv[0]), int(svv[1]))
        self.h = self.L.or_assemble_svv(mesh.h, _pi(self.f2v), ng, c_mass, c_lap,
                                        int(bool(quirk)), _pd(sv), svc, svn)
        self.n = ng

    class _View(ctypes.Structure):
        _fields_ = [("n", _int), ("nnz", _int), ("rowptr", _I), ("col", _I), ("val", _D),
                    ("lift", _D)]

    def arrays(self):
        v = ctypes.cast(self.h, ctypes.POINTER(self._View)).contents
        rowptr = np.ctypeslib.as_array(v.rowptr, shape=(v.n + 1,)).copy()
        col = np.ctypeslib.as_array(v.col, shape=(max(v.nnz, 1),))[: v.nnz].copy()
        val = np.ctypeslib.as_array(v.val, shape=(max(v.nnz, 1),))[: v.nnz].copy()
        lift = np.ctypeslib.as_array(v.lift, shape=(max(v.n, 1),))[: v.n].copy()
        return rowptr, col, val, lift

    def matvec(self, x, nthreads=1):
        x = _f64(x)
        y = np.zeros(self.n)
        self.L.or_csr_matvec(self.h, _pd(x), _pd(y), nthreads)
        return y

    def pcg(self, b, rtol=1e-10, atol=1e-50, dtol=1e5, max_it=10000, norm_type=0,
            remove_null_space=False, nthreads=1):
        b = _f64(b)
        x = np.zeros(self.n)
        its, rn, rn0 = _int(0), _dbl(0), _dbl(0)
        reason = self.L.or_pcg(self.h, _pd(b), _pd(x), rtol, atol, dtol, max_it, norm_type,
                               int(bool(remove_null_space)), nthreads, ctypes.byref(its),
                               ctypes.byref(rn), ctypes.byref(rn0))
        return x, {"reason": reason, "its": its.value, "rnorm": rn.value, "rnorm0": rn0.value}

    def close(self):
        if self.h:
            self.L.or_csr_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def assemble_rhs(mesh: Mesh, f2v, ng, rhs_vals):
    f = np.zeros(ng)
    f2v = np.ascontiguousarray(f2v, dtype=np.int32)
    mesh.L.or_assemble_rhs(mesh.h, _pi(f2v), ng, _pd(_f64(rhs_vals)), _pd(f))
    return f


def update_field(mesh: Mesh, v2f, x, vals):
    vals = _f64(vals).copy()
    v2f = np.ascontiguousarray(v2f, dtype=np.int32)
    mesh.L.or_update_field(mesh.h, _pi(v2f), len(v2f), _pd(_f64(x)), _pd(vals))
    return vals


def helmholtz_solve(mesh: Mesh, sol_vals, rhs_vals, c, nu, dt, bcs=(False, False, False, False),
                    quirk=True, rtol=1e-10, atol=1e-50, max_it=10000, norm_type=0,
                    remove_null_space=False, nthreads=1, poisson=False, project_rhs=False,
                    svv_cutoff=0):
    """HelmholtzEqn (src/linsys/HelmholtzEqn.cpp:43-158) or, with poisson=True,
    PoissonEqn(c) (src/linsys/PoissonEqn.cpp:30-134), solved by the restated
    Jacobi-PCG; a Helmholtz system with svv_cutoff != 0 adds the SVV
    operator SVV(dt, svv_cutoff) as HelmholtzEqn does (src/linsys/
    HelmholtzEqn.cpp:71). project_rhs (with remove_null_space) first replaces the
    assembled right-hand side b by b - (sum b / sum d) d, d the matrix
    diagonal: the consistent system that Jacobi CG with the null space
    projected out of its preconditioned residuals approaches when b is off
    the operator's range. Returns the updated solution field and the solver
    stats."""
    f2v, v2f = mesh.bcs_maps(*bcs)
    ng = len(v2f)
    if poisson:
        A = CSR(mesh, f2v, ng, 0.0, c, quirk, sol_vals)
    else:
        A = CSR(mesh, f2v, ng, c, nu * dt, quirk, sol_vals,
                svv=(dt, svv_cutoff) if svv_cutoff else None)
    f = assemble_rhs(mesh, f2v, ng, rhs_vals)
    rowptr, col, val, lift = A.arrays()
    f = f + lift
    if project_rhs and remove_null_space:
        d = np.zeros(ng)
        for k in range(ng):
            row = slice(rowptr[k], rowptr[k + 1])
            d[k] = val[row][col[row] == k].sum()
        f = f - (f.sum() / d.sum()) * d
    x, stats = A.pcg(f, rtol=rtol, atol=atol, max_it=max_it, norm_type=norm_type,
                     remove_null_space=remove_null_space, nthreads=nthreads)
    out = update_field(mesh, v2f, x, sol_vals)
    A.close()
    stats["x"] = x
    stats["b"] = f
    return out, stats


class QG2:
    """TwoLayerQGEqn (src/qg/TwoLayerQGEqn.cpp:17-433) restated over the
    oracle's pieces: GenPV, GenVel (InterpDerivsGlobal at the vertices), the
    restated SL advection, Helmholtz/Poisson solves by the restated CSR +
    Jacobi-PCG, and SolveQ as the assembled DissipationRHS divided by the
    diagonal PV mass. Follows the reference's step as written (first order:
    SolveQ for layer 1 only; dissipation of both layers with tau1; PV mass
    x 1.5 from the first second-order step). Arrays in the reference's vertex
    order. TEST INFRASTRUCTURE ONLY."""

    def __init__(self, mesh: Mesh, bcs, psi1, omega1, psi2, omega2, F1, F2, beta, E2, r, nu,
                 tau_e, dt, quirk=False, rtol=1e-12, nthreads=1):
        self.m, self.bcs, self.quirk, self.rtol = mesh, tuple(bcs), quirk, rtol
        self.nthreads = nthreads
        self.F1, self.F2, self.beta, self.E2, self.r, self.nu, self.dt = F1, F2, beta, E2, r, nu, dt
        self.psi1, self.omega1 = _f64(psi1).copy(), _f64(omega1).copy()
        self.psi2, self.omega2 = _f64(psi2).copy(), _f64(omega2).copy()
        self.tau_e = _f64(tau_e).copy()
        self.X = mesh.verts()
        self.y = self.X[:, 1].copy()
        self.f2v, self.v2f = mesh.bcs_maps(*bcs)
        self.tau1 = self.psi1 - self.psi2
        self.chi1 = self.psi1 + self.psi2
        self.tau2, self.chi2 = self.tau1.copy(), self.chi1.copy()
        self.alpha1 = self.gen_pv(self.omega1, self.psi1, self.psi2, F1)
        self.alpha2 = self.gen_pv(self.omega2, self.psi2, self.psi1, F2)
        self.a_mass, self.second = 1.0, False

    def gen_pv(self, omega, psi_i, psi_j, F):
        return omega + F * (psi_j - psi_i) + self.beta * self.y

    def gen_vel(self, psi):
        d = self.m.interp_derivs_global(psi, self.X)
        return np.stack([-d[:, 1], d[:, 0]], 1)

    def helm(self, sol, rhs):
        return helmholtz_solve(self.m, sol, rhs, -(self.F1 + self.F2), -1.0, 1.0, self.bcs,
                               quirk=self.quirk, rtol=self.rtol, nthreads=self.nthreads)[0]

    def fish(self, sol, rhs):
        return helmholtz_solve(self.m, sol, rhs, -1.0, 0.0, 0.0, self.bcs, quirk=self.quirk,
                               rtol=self.rtol, poisson=True, nthreads=self.nthreads)[0]

    def solve_q(self, alpha_hat, om_hat, rF, Ei, alpha):
        ng = len(self.v2f)
        f2v = np.ascontiguousarray(self.f2v, dtype=np.int32)
        f, d = np.zeros(ng), np.zeros(ng)
        self.m.L.or_dissipation_rhs(self.m.h, _pi(f2v), ng, self.dt, _pd(_f64(alpha_hat)),
                                    _pd(_f64(self.tau1)), _pd(_f64(om_hat)), _pd(self.tau_e),
                                    rF, Ei, self.nu, _pd(f))
        self.m.L.or_mass_diag(self.m.h, _pi(f2v), ng, self.a_mass, _pd(d))
        return update_field(self.m, self.v2f, f / d, alpha)

    def invert(self, a1, a2, tau, chi, cb_fish, cb_update):
        tau = self.helm(tau, a1 - a2)
        chi = self.fish(chi, a1 + a2 + (self.F1 - self.F2) * tau - cb_fish * self.y)
        p1, p2 = 0.5 * (tau + chi), 0.5 * (chi - tau)
        o1 = a1 - self.F1 * (p2 - p1) - cb_update * self.y
        o2 = a2 - self.F2 * (p1 - p2) - cb_update * self.y
        return tau, chi, p1, p2, o1, o2

    def step(self, prev=None):
        """One TwoLayerQGEqn::Solve; prev = (psi1, omega1, psi2, omega2) of
        the previous step (second order) or None (first order). Returns the
        new prev tuple (the fields before this step) for second order."""
        m, dt, b = self.m, self.dt, self.beta
        if prev is None:
            vel1, vel2 = self.gen_vel(self.psi1), self.gen_vel(self.psi2)
            self.alpha1 = self.gen_pv(self.omega1, self.psi1, self.psi2, self.F1)
            self.alpha2 = self.gen_pv(self.omega2, self.psi2, self.psi1, self.F2)
            a1h = m.advect(self.alpha1, vel1, dt, nthreads=self.nthreads)
            a2h = m.advect(self.alpha2, vel2, dt, nthreads=self.nthreads)
            self.tau1, self.chi1, _, _, o1h, _ = self.invert(a1h, a2h, self.tau1, self.chi1,
                                                             2.0 * b, b)
            self.alpha1 = self.solve_q(a1h, o1h, self.r * self.F1, 0.0, self.alpha1)
            (self.tau2, self.chi2, self.psi1, self.psi2, self.omega1,
             self.omega2) = self.invert(self.alpha1, self.alpha2, self.tau2, self.chi2, 2.0 * b, b)
            return None
        if not self.second:
            self.a_mass, self.second = 1.5, True
        p1p, o1p, p2p, o2p = [_f64(v).copy() for v in prev]
        saved = (self.psi1.copy(), self.omega1.copy(), self.psi2.copy(), self.omega2.copy())
        a = 1.5
        vel1, vel2 = self.gen_vel(self.psi1), self.gen_vel(self.psi2)
        vel1p, vel2p = self.gen_vel(p1p), self.gen_vel(p2p)
        self.alpha1 = self.gen_pv(self.omega1, self.psi1, self.psi2, self.F1)
        self.alpha2 = self.gen_pv(self.omega2, self.psi2, self.psi1, self.F2)
        a1p = self.gen_pv(o1p, p1p, p2p, self.F1)
        a2p = self.gen_pv(o2p, p2p, p1p, self.F2)
        a1h = m.advect(self.alpha1, vel1, dt, a1p, vel1p, nthreads=self.nthreads)
        a2h = m.advect(self.alpha2, vel2, dt, a2p, vel2p, nthreads=self.nthreads)
        self.tau1, self.chi1, _, _, o1h, o2h = self.invert(a1h, a2h, self.tau1, self.chi1,
                                                           a * 2.0 * b, a * b)
        self.alpha1 = self.solve_q(a1h, o1h, self.r * self.F1, 0.0, self.alpha1)
        self.alpha2 = self.solve_q(a2h, o2h, -self.r * self.F2, self.E2, self.alpha2)
        (self.tau2, self.chi2, self.psi1, self.psi2, self.omega1,
         self.omega2) = self.invert(self.alpha1, self.alpha2, self.tau2, self.chi2, 2.0 * b, b)
        return saved


class NS:
    """NavierStokesEqn (src/ns/NavierStokesEqn.cpp:23-147) restated over the
    oracle's pieces: SL advection of the velocity by itself, the divergence of
    the advected velocity and the pressure gradient by InterpDerivsGlobal at
    the vertices, the pressure PoissonEqn(-dt) with the constant null space
    removed (its right-hand side projected onto the operator's range first,
    see helmholtz_solve's project_rhs) and the viscous HelmholtzEqn(c, nu,
    dt) per velocity component
    (the reference's interleaved 2-component matrix is block diagonal per
    component: src/base/Operator.cpp:67-79, :161-172), all by the restated
    CSR + Jacobi-PCG. The second-order step scales the divergence by 1.5 and
    10.0 and uses c = 1.5, as the reference writes it. bcs_u, bcs_v are the
    (bottom, top, left, right) Dirichlet flags of each velocity component;
    the pressure has none. TEST INFRASTRUCTURE ONLY."""

    def __init__(self, mesh: Mesh, bcs_u, bcs_v, dt, quirk=False, rtol=1e-12):
        self.m, self.dt, self.quirk, self.rtol = mesh, dt, quirk, rtol
        self.bcs = (tuple(bcs_u), tuple(bcs_v))
        self.X = mesh.verts()

    def derivs(self, vals):
        return self.m.interp_derivs_global(vals, self.X)

    def step(self, vel, pres, prev_vel, nu, svv_cutoff=0):
        """One Solve(velocity, pressure, prevVel, nu, svvCutoff); returns
        (velocity, pressure, stats) after the step."""
        m, dt = self.m, self.dt
        vel, pres = _f64(vel).copy(), _f64(pres).copy()
        second = prev_vel is not None
        if second:
            sl = m.advect(vel, vel, dt, _f64(prev_vel), _f64(prev_vel))
        else:
            sl = m.advect(vel, vel, dt)
        div = self.derivs(np.ascontiguousarray(sl[:, 0]))[:, 0] + \
            self.derivs(np.ascontiguousarray(sl[:, 1]))[:, 1]
        if second:
            div = div * 1.5 * 10.0
        # the vertex divergence is off the Neumann operator's range by a little:
        # solve the consistent system the reference's CG approaches
        pres, sp = helmholtz_solve(m, pres, div, -dt, 0.0, 0.0, quirk=self.quirk, rtol=self.rtol,
                                   remove_null_space=True, poisson=True, project_rhs=True)
        dp = self.derivs(pres)
        step2 = sl - dt * dp
        c = 1.5 if second else 1.0
        stats = [sp]
        for d in range(2):
            col, st = helmholtz_solve(m, np.ascontiguousarray(vel[:, d]),
                                      np.ascontiguousarray(step2[:, d]), c, nu, dt, self.bcs[d],
                                      quirk=self.quirk, rtol=self.rtol, svv_cutoff=svv_cutoff)
            vel[:, d] = col
            stats.append(st)
        return vel, pres, stats
