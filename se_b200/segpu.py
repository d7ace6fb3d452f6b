"""Python mirror of SE's hot-path classes over the segpu C-ABI.

The classes keep the reference's names, constructor arguments and methods,
so code written against SE's ``src/base`` / ``src/linsys`` reads the same:

=====================  =================================================
reference (C++)        here
=====================  =================================================
``Mesh``               :class:`Mesh`   (src/base/Mesh.h:4-37)
``BCs``                :class:`BCs`    (src/base/BCs.h:1-22)
``Field``              :class:`Field`  (src/base/Field.h:5-31)
``Advector``           :class:`Advector` (src/base/Advector.h:1-28)
``HelmholtzEqn``       :class:`HelmholtzEqn` (src/linsys/HelmholtzEqn.h:1-22)
``PoissonEqn``         :class:`PoissonEqn` (src/linsys/PoissonEqn.h:1-19)
``CalcTimeStep``       :func:`CalcTimeStep` (src/base/Utils.cpp:23-40)
``FieldError``         :func:`FieldError` (src/base/Utils.cpp:232-254)
=====================  =================================================

Everything runs on the GPU through ``libsegpu.so``; a missing library or a
missing CUDA device raises :class:`SEError` -- there is no CPU fallback.
Where the reference calls ``exit(1)`` on a configuration error, this layer
raises :class:`SEError` with the library's message.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsegpu.so")

SE_OK = 0
SE_ERR_ARG = -1
SE_ERR_OOM = -2
SE_ERR_CUDA = -3
SE_ERR_UNSUPPORTED = -4
SE_ERR_NOT_CONVERGED = -5
SE_ERR_TIMEOUT = -6
SE_ERR_DOMAIN = -7

NORM_PRECONDITIONED, NORM_UNPRECONDITIONED, NORM_NATURAL = 0, 1, 2
MODE_REFERENCE, MODE_EXACT = 0, 1
PREC_FP64, PREC_MIXED, PREC_BF16, PREC_FP16, PREC_FP64_TC = 0, 1, 2, 3, 4
METHOD_CG, METHOD_FDM = 0, 1

KSP_REASONS = {2: "CONVERGED_RTOL", 3: "CONVERGED_ATOL", -3: "DIVERGED_ITS",
               -4: "DIVERGED_DTOL", -5: "DIVERGED_BREAKDOWN", -8: "DIVERGED_INDEFINITE_PC",
               -9: "DIVERGED_NANORINF", -10: "DIVERGED_INDEFINITE_MAT"}


class SEError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"segpu error {code}: {msg}")
        self.code = code


class SolverOpts(ctypes.Structure):
    _fields_ = [("rtol", ctypes.c_double), ("atol", ctypes.c_double),
                ("dtol", ctypes.c_double), ("max_it", ctypes.c_int),
                ("norm_type", ctypes.c_int), ("mode", ctypes.c_int),
                ("precision", ctypes.c_int), ("inner_max_it", ctypes.c_int),
                ("inner_rtol", ctypes.c_double), ("method", ctypes.c_int)]


class SolveStats(ctypes.Structure):
    _fields_ = [("reason", ctypes.c_int), ("its", ctypes.c_int), ("outer_its", ctypes.c_int),
                ("rnorm", ctypes.c_double), ("rnorm0", ctypes.c_double),
                ("kernel_ms", ctypes.c_double)]

    def as_dict(self):
        return {"reason": self.reason, "its": self.its, "outer_its": self.outer_its,
                "rnorm": self.rnorm, "rnorm0": self.rnorm0, "kernel_ms": self.kernel_ms}


class Request(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("nEls", ctypes.c_int * 2), ("N", ctypes.c_int),
                ("min", ctypes.c_double * 2), ("max", ctypes.c_double * 2),
                ("periodic", ctypes.c_int * 2), ("bcs", ctypes.c_int * 4),
                ("c", ctypes.c_double), ("nu", ctypes.c_double), ("dt", ctypes.c_double),
                ("poisson", ctypes.c_int), ("opts", SolverOpts), ("steps", ctypes.c_int),
                ("sl_dt", ctypes.c_double), ("in_", ctypes.c_void_p), ("aux", ctypes.c_void_p),
                ("out", ctypes.c_void_p)]


class Result(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("reason", ctypes.c_int), ("its", ctypes.c_int),
                ("queued_ms", ctypes.c_double), ("latency_ms", ctypes.c_double),
                ("error", ctypes.c_char * 160)]


REQ_HELMHOLTZ, REQ_ADVECT = 0, 1

_lib = None
_vp = ctypes.c_void_p
_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)

# name -> argtypes for every entry point declared in include/segpu.h
SIGNATURES = {
    "se_last_error": [], "se_version": [], "se_set_stream": [_vp], "se_synchronize": [],
    "se_mesh_create": [_I, ctypes.c_int, _D, _D, _I, ctypes.POINTER(_vp)],
    "se_mesh_destroy": [_vp], "se_mesh_sizes": [_vp, _I, _I], "se_mesh_verts": [_vp, _D],
    "se_mesh_gll": [_vp, _D, _D, _D],
    "se_mesh_global_to_local": [_vp, _D, ctypes.c_int, _I, _D],
    "se_bcs_create": [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                      ctypes.POINTER(_vp)],
    "se_bcs_destroy": [_vp], "se_bcs_vec_size": [_vp, _I], "se_bcs_maps": [_vp, _I, _I],
    "se_field_create": [_vp, ctypes.c_int, _vp, ctypes.POINTER(_vp)],
    "se_field_destroy": [_vp], "se_field_upload": [_vp, _D], "se_field_download": [_vp, _D],
    "se_field_device_ptr": [_vp, ctypes.POINTER(_vp)], "se_field_copy": [_vp, _vp],
    "se_field_periodic_update": [_vp],
    "se_field_integrate": [_vp, ctypes.c_int, ctypes.c_int, _D],
    "se_field_interp_global": [_vp, _D, ctypes.c_int, _D],
    "se_advector_create": [_vp, _vp, _vp, _vp, ctypes.POINTER(_vp)],
    "se_advector_destroy": [_vp], "se_advect": [_vp, ctypes.c_double],
    "se_advector_field_sl": [_vp, ctypes.POINTER(_vp)],
    "se_advector_departures": [_vp, _I, _D],
    "se_solver_opts_default": [ctypes.POINTER(SolverOpts)],
    "se_solver_opts_parse": [ctypes.POINTER(SolverOpts), ctypes.c_char_p, ctypes.c_char_p],
    "se_helmholtz_create": [_vp, _vp, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                            ctypes.c_int, ctypes.POINTER(SolverOpts), ctypes.POINTER(_vp)],
    "se_poisson_create": [_vp, _vp, ctypes.c_double, ctypes.POINTER(SolverOpts),
                          ctypes.POINTER(_vp)],
    "se_linsys_destroy": [_vp], "se_linsys_set_opts": [_vp, ctypes.POINTER(SolverOpts)],
    "se_linsys_assemble": [_vp],
    "se_linsys_solve": [_vp, ctypes.c_int, ctypes.POINTER(SolveStats)],
    "se_linsys_solve_batch": [ctypes.POINTER(_vp), ctypes.c_int, ctypes.c_int,
                              ctypes.POINTER(SolveStats)],
    "se_linsys_solve_async": [_vp, ctypes.c_int],
    "se_linsys_solve_finish": [_vp, ctypes.POINTER(SolveStats)],
    "se_linsys_apply": [_vp, _vp, _vp], "se_field_gen_vel": [_vp, _vp], "se_field_save": [_vp, ctypes.c_char_p, ctypes.c_int], "se_field_read": [_vp, ctypes.c_char_p, ctypes.c_int], "se_linsys_fdm_apply": [_vp, _vp, _vp], "se_linsys_fdm_apply_prec": [_vp, ctypes.c_int, _vp, _vp], "se_linsys_residual": [_vp, _vp, _vp, _vp], "se_linsys_apply_low": [_vp, ctypes.c_int, _vp, _vp], "se_linsys_diagonal": [_vp, _vp],
    "se_linsys_vec_size": [_vp, _I],
    "se_calc_time_step": [_vp, ctypes.c_double, _D],
    "se_field_error": [_vp, _vp, ctypes.c_int, ctypes.c_int, _D],
    "se_server_create": [ctypes.c_int, ctypes.c_double, ctypes.POINTER(_vp)],
    "se_server_submit": [_vp, ctypes.POINTER(Request), ctypes.POINTER(ctypes.c_longlong)],
    "se_server_wait": [_vp, ctypes.c_longlong, ctypes.POINTER(Result)],
    "se_server_destroy": [_vp],
    "se_qg2_create": [_vp, _vp, _vp, _vp] + [ctypes.c_double] * 6 +
                     [_vp, ctypes.c_double, ctypes.POINTER(SolverOpts), ctypes.POINTER(_vp)],
    "se_qg2_solve": [_vp, _vp, _vp, _vp, _vp], "se_qg2_destroy": [_vp],
    "se_ns_create": [_vp, _vp, _vp, _vp, ctypes.c_double, ctypes.POINTER(SolverOpts),
                     ctypes.POINTER(_vp)],
    "se_ns_solve": [_vp, _vp, _vp, _vp, ctypes.c_double, ctypes.c_int],
    "se_ns_stats": [_vp, ctypes.POINTER(SolveStats)], "se_ns_destroy": [_vp],
    "se_field_download_async": [_vp, _D],
    "se_mesh_save": [_vp, ctypes.c_char_p], "se_write_xdmf_header": [ctypes.c_int],
    "se_write_xdmf_footer": [ctypes.c_int], "se_write_xdmf_temporal": [ctypes.c_int, ctypes.c_int],
    "se_write_xdmf": [ctypes.POINTER(_vp), ctypes.POINTER(ctypes.c_char_p), ctypes.c_int,
                      ctypes.c_char_p, ctypes.c_int, ctypes.c_double, ctypes.c_double],
    "se_helmholtz_solve_noalloc": [_I, ctypes.c_int, _D, _D, _I, _I, ctypes.c_double,
                                   ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                   ctypes.POINTER(SolverOpts), ctypes.c_int, _vp, _vp,
                                   ctypes.POINTER(SolveStats)],
}


def load_library(path: str = LIB_PATH):
    """Load libsegpu.so (raises if it is missing: the GPU path has no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise SEError(SE_ERR_CUDA, f"{path} is missing: run `python -m se_b200.build`")
    L = ctypes.CDLL(path)
    for name, args in SIGNATURES.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = ctypes.c_char_p if name in ("se_last_error", "se_version") else ctypes.c_int
    _lib = L
    return L


def _check(rc: int):
    if rc != SE_OK:
        msg = _lib.se_last_error().decode()
        raise SEError(rc, msg)


def _pd(a):
    return a.ctypes.data_as(_D)


def _pi(a):
    return a.ctypes.data_as(_I)


def set_stream(stream_ptr: int | None):
    """Queue library work on a cudaStream_t (e.g. torch.cuda.current_stream().cuda_stream)."""
    _check(load_library().se_set_stream(_vp(stream_ptr or 0)))


def synchronize():
    _check(load_library().se_synchronize())


class Mesh:
    """Mesh(name, nEls, "legendre", N, min, max, periodic) (src/base/Mesh.h:6)."""

    def __init__(self, name, nEls, elType, N, min, max, periodic):
        if elType != "legendre":
            raise SEError(SE_ERR_UNSUPPORTED, f"element type {elType!r}: only 'legendre' is built")
        L = load_library()
        self.name = name
        self.N = int(N)
        self.nEls = [int(nEls[0]), int(nEls[1])]
        self.min = [float(min[0]), float(min[1])]
        self.max = [float(max[0]), float(max[1])]
        self.periodic = [bool(periodic[0]), bool(periodic[1])]
        ne = (ctypes.c_int * 2)(*self.nEls)
        mn = (ctypes.c_double * 2)(*self.min)
        mx = (ctypes.c_double * 2)(*self.max)
        pe = (ctypes.c_int * 2)(*[int(p) for p in self.periodic])
        h = _vp()
        _check(L.se_mesh_create(ne, self.N, mn, mx, pe, ctypes.byref(h)))
        self._h = h
        nv = (ctypes.c_int * 2)()
        nt = ctypes.c_int()
        _check(L.se_mesh_sizes(h, nv, ctypes.byref(nt)))
        self.nVerts = [nv[0], nv[1]]
        self.nVertsTotal = nt.value
        self.nElsTotal = self.nEls[0] * self.nEls[1]
        self.dx = [(self.max[k] - self.min[k]) / self.nEls[k] for k in range(2)]

    @property
    def verts(self):
        v = np.zeros((self.nVertsTotal, 2))
        _check(_lib.se_mesh_verts(self._h, _pd(v)))
        return v

    def Save(self):
        """Mesh::Save (src/base/Mesh.cpp:366-489): <name>.seb in the working
        directory (raw binary in place of <name>.h5)."""
        _check(_lib.se_mesh_save(self._h, self.name.encode()))

    def gll(self):
        n = self.N + 1
        a, w, d = np.zeros(n), np.zeros(n), np.zeros(n * n)
        _check(_lib.se_mesh_gll(self._h, _pd(a), _pd(w), _pd(d)))
        return a, w, d.reshape(n, n)

    def GlobalToLocal(self, pts):
        pts = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, 2)
        el = np.zeros(len(pts), dtype=np.int32)
        lc = np.zeros_like(pts)
        _check(_lib.se_mesh_global_to_local(self._h, _pd(pts), len(pts), _pi(el), _pd(lc)))
        return el, lc

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.se_mesh_destroy(self._h)
            self._h = None


class BCs:
    """BCs(bottom, top, left, right, mesh, 0) (src/base/BCs.h:3). With one
    flag per side it is the scalar constructor (src/base/BCs.cpp:14-); with a
    pair of flags per side it is the 2-component constructor
    (src/base/BCs.cpp:175-), held as one scalar BCs per component in
    ``components`` (used by NavierStokesEqn's viscous step)."""

    def __init__(self, bcBottom, bcTop, bcLeft, bcRight, mesh: Mesh, vecOffset=0):
        if vecOffset != 0:
            raise SEError(SE_ERR_UNSUPPORTED, "vecOffset != 0 (block systems) is not built")
        sides = (bcBottom, bcTop, bcLeft, bcRight)
        self.components = None
        if any(isinstance(b, (list, tuple, np.ndarray)) for b in sides):
            pairs = [tuple(b) if isinstance(b, (list, tuple, np.ndarray)) else (b, b)
                     for b in sides]
            if any(len(p) != 2 for p in pairs):
                raise SEError(SE_ERR_ARG, "per-component BCs need two flags per side")
            self.components = tuple(BCs(*(bool(p[d]) for p in pairs), mesh) for d in range(2))
            self._h, self.mesh = None, mesh
            self.size = [c.vecSize for c in self.components]
            self.vecSize = sum(self.size)
            return
        h = _vp()
        _check(load_library().se_bcs_create(mesh._h, int(bcBottom), int(bcTop), int(bcLeft),
                                            int(bcRight), ctypes.byref(h)))
        self._h, self.mesh = h, mesh
        n = ctypes.c_int()
        _check(_lib.se_bcs_vec_size(h, ctypes.byref(n)))
        self.vecSize = n.value

    def maps(self):
        if self.components is not None:
            raise SEError(SE_ERR_UNSUPPORTED, "maps of per-component BCs: use components[d]")
        f2v = np.zeros(self.mesh.nVertsTotal, dtype=np.int32)
        v2f = np.zeros(self.vecSize, dtype=np.int32)
        _check(_lib.se_bcs_maps(self._h, _pi(f2v), _pi(v2f)))
        return f2v, v2f

    @property
    def fieldToVecMap(self):
        return self.maps()[0]

    @property
    def vecToFieldMap(self):
        return self.maps()[1]

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.se_bcs_destroy(self._h)
            self._h = None


class Field:
    """Field(name, mesh, nDofs, bcs) (src/base/Field.h:7). ``vals`` reads or
    writes the whole [nVertsTotal][nDofs] array on the GPU."""

    def __init__(self, name, mesh: Mesh, nDofs, bcs: BCs | None, _handle=None, _owner=None):
        self.name, self.mesh, self.nDofs, self.bcs = name, mesh, int(nDofs), bcs
        self._owner = _owner
        if _handle is not None:
            self._h, self._borrowed = _handle, True
            return
        h = _vp()
        _check(load_library().se_field_create(mesh._h, self.nDofs, bcs._h if bcs else None,
                                              ctypes.byref(h)))
        self._h, self._borrowed = h, False

    def _shape(self):
        n = self.mesh.nVertsTotal
        return (n,) if self.nDofs == 1 else (n, self.nDofs)

    @property
    def vals(self) -> np.ndarray:
        out = np.zeros(self._shape())
        _check(_lib.se_field_download(self._h, _pd(out)))
        return out

    @vals.setter
    def vals(self, v):
        a = np.ascontiguousarray(np.broadcast_to(np.asarray(v, dtype=np.float64), self._shape()))
        _check(_lib.se_field_upload(self._h, _pd(a)))

    def device_ptr(self) -> int:
        p = _vp()
        _check(_lib.se_field_device_ptr(self._h, ctypes.byref(p)))
        return p.value

    def Copy(self, field: "Field"):
        _check(_lib.se_field_copy(self._h, field._h))

    def Save(self, timeStep: int, name: str | None = None):
        """Field::Save: writes "<name>.<timeStep:05>.seb" (raw binary; see se_field_save)."""
        _check(_lib.se_field_save(self._h, (name or self.name).encode(), int(timeStep)))

    def Read(self, timeStep: int, name: str | None = None):
        """Field::Read of a file written by Save."""
        _check(_lib.se_field_read(self._h, (name or self.name).encode(), int(timeStep)))

    def PeriodicUpdate(self):
        _check(_lib.se_field_periodic_update(self._h))

    def Integrate(self, dof=0, average=False):
        out = ctypes.c_double()
        _check(_lib.se_field_integrate(self._h, dof, int(average), ctypes.byref(out)))
        return out.value

    def InterpGlobal(self, pts):
        pts = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, 2)
        out = np.zeros((len(pts), self.nDofs))
        _check(_lib.se_field_interp_global(self._h, _pd(pts), len(pts), _pd(out)))
        return out

    def SetICFunc(self, dof, func):
        """Field::SetICFunc (src/base/Field.cpp:226-230) with a vectorised func(x, y)."""
        X = self.mesh.verts
        v = self.vals
        vals = func(X[:, 0], X[:, 1])
        if self.nDofs == 1:
            v = np.asarray(vals, dtype=np.float64) + 0 * v
        else:
            v[:, dof] = vals
        self.vals = v

    def __del__(self):
        if getattr(self, "_h", None) and not self._borrowed and _lib is not None:
            _lib.se_field_destroy(self._h)
            self._h = None


class Advector:
    """Advector(field, velocity[, fieldMinusOne, velMinusOne]) (src/base/Advector.h:3-4)."""

    def __init__(self, field: Field, velocity: Field, fieldMinusOne: Field | None = None,
                 velMinusOne: Field | None = None):
        h = _vp()
        _check(load_library().se_advector_create(
            field._h, velocity._h, fieldMinusOne._h if fieldMinusOne else None,
            velMinusOne._h if velMinusOne else None, ctypes.byref(h)))
        self._h = h
        self.field, self.velocity = field, velocity
        self.fieldMinusOne, self.velMinusOne = fieldMinusOne, velMinusOne
        self.secondOrder = fieldMinusOne is not None
        sl = _vp()
        _check(_lib.se_advector_field_sl(h, ctypes.byref(sl)))
        self.fieldSL = Field(f"{field.name}-SL", field.mesh, field.nDofs, field.bcs,
                             _handle=sl, _owner=self)

    def Advect(self, dt):
        _check(_lib.se_advect(self._h, float(dt)))

    def record_departures(self):
        """Enable recording of departure elements/points for the next Advect."""
        rc = _lib.se_advector_departures(self._h, None, None)
        if rc not in (SE_OK, SE_ERR_ARG):
            _check(rc)

    def departures(self):
        """(elements, points) of the last Advect; second order stacks x1 then x2."""
        k = 2 if self.secondOrder else 1
        n = self.field.mesh.nVertsTotal
        el = np.zeros(k * n, dtype=np.int32)
        xy = np.zeros((k * n, 2))
        _check(_lib.se_advector_departures(self._h, _pi(el), _pd(xy)))
        return el, xy

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.se_advector_destroy(self._h)
            self._h = None


def solver_opts(prefix: str = "", options: str = "", **kw) -> SolverOpts:
    """Default solver options, a PETSc-style options string for one prefix,
    then keyword overrides (rtol, atol, dtol, max_it, norm_type, mode, precision)."""
    o = SolverOpts()
    _check(load_library().se_solver_opts_default(ctypes.byref(o)))
    if options:
        _check(_lib.se_solver_opts_parse(ctypes.byref(o), prefix.encode(), options.encode()))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


class _LinSys:
    _h = None

    def Assemble(self):
        _check(_lib.se_linsys_assemble(self._h))

    def set_opts(self, opts: SolverOpts):
        self.opts = opts
        _check(_lib.se_linsys_set_opts(self._h, ctypes.byref(opts)))

    def _solve(self, removeNullSpace: bool, raise_on_diverge: bool, projectRHS: bool = False):
        st = SolveStats()
        null = (2 if projectRHS else 1) if removeNullSpace else 0
        rc = _lib.se_linsys_solve(self._h, null, ctypes.byref(st))
        if rc == SE_ERR_NOT_CONVERGED and not raise_on_diverge:
            rc = SE_OK
        _check(rc)
        self.stats = st.as_dict()
        return self.stats

    def solve_async(self, removeNullSpace: bool = False, projectRHS: bool = False):
        """Queue the solve on the library's stream (se_linsys_solve_async); FDM
        solves return at once, CG solves complete before returning."""
        null = (2 if projectRHS else 1) if removeNullSpace else 0
        _check(_lib.se_linsys_solve_async(self._h, null))

    def solve_finish(self, raise_on_diverge: bool = False):
        """Wait for a queued solve and return its statistics."""
        st = SolveStats()
        rc = _lib.se_linsys_solve_finish(self._h, ctypes.byref(st))
        if rc == SE_ERR_NOT_CONVERGED and not raise_on_diverge:
            rc = SE_OK
        _check(rc)
        self.stats = st.as_dict()
        return self.stats

    @property
    def vecSize(self):
        n = ctypes.c_int()
        _check(_lib.se_linsys_vec_size(self._h, ctypes.byref(n)))
        return n.value

    def apply(self, x_ptr: int, y_ptr: int):
        """y = A x on device pointers of vecSize doubles."""
        _check(_lib.se_linsys_apply(self._h, _vp(x_ptr), _vp(y_ptr)))

    def residual(self, x_ptr: int, b_ptr: int, r_ptr: int):
        """r = b - A x in double-double, rounded once (device pointers)."""
        _check(_lib.se_linsys_residual(self._h, _vp(x_ptr), _vp(b_ptr), _vp(r_ptr)))

    def fdm_apply(self, r_ptr: int, x_ptr: int, precision: int = PREC_FP64):
        """x = A^{-1} r by the fast-diagonalization transforms (device pointers):
        FP64 products, or (PREC_MIXED) TF32 hi/lo products on the tensor cores."""
        if precision == PREC_FP64:
            _check(_lib.se_linsys_fdm_apply(self._h, _vp(r_ptr), _vp(x_ptr)))
        else:
            _check(_lib.se_linsys_fdm_apply_prec(self._h, int(precision), _vp(r_ptr), _vp(x_ptr)))

    def apply_low(self, x_ptr: int, y_ptr: int, precision: int = PREC_BF16):
        """y (FP32) = A x for x of vecSize BF16 (or FP16) values; device pointers."""
        _check(_lib.se_linsys_apply_low(self._h, int(precision), _vp(x_ptr), _vp(y_ptr)))

    def diagonal(self, d_ptr: int):
        _check(_lib.se_linsys_diagonal(self._h, _vp(d_ptr)))

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.se_linsys_destroy(self._h)
            self._h = None


class HelmholtzEqn(_LinSys):
    """HelmholtzEqn(solField, rhsField, c, nu, dt, svvCutoff)
    (src/linsys/HelmholtzEqn.h:3): A = c*Mass + nu*dt*Laplacian."""

    def __init__(self, solField: Field, rhsField: Field | None, c, nu, dt, svvCutoff=0,
                 opts: SolverOpts | None = None):
        self.solField, self.rhsField = solField, rhsField
        self.c, self.nu, self.dt = float(c), float(nu), float(dt)
        self.opts = opts or solver_opts()
        h = _vp()
        _check(load_library().se_helmholtz_create(
            solField._h, rhsField._h if rhsField else None, self.c, self.nu, self.dt,
            int(svvCutoff), ctypes.byref(self.opts), ctypes.byref(h)))
        self._h = h

    def Solve(self, name: str = "helm_", removeNullSpace: bool = False, options: str = "",
              raise_on_diverge: bool = False, projectRHS: bool = False):
        """HelmholtzEqn::Solve(name, removeNullSpace); ``options`` is the PETSc
        options string consulted under prefix ``name``; projectRHS (with
        removeNullSpace) solves the consistent system (se_linsys_solve mode 2)."""
        if options:
            o = SolverOpts.from_buffer_copy(self.opts)
            _check(_lib.se_solver_opts_parse(ctypes.byref(o), name.encode(), options.encode()))
            self.set_opts(o)
        return self._solve(removeNullSpace, raise_on_diverge, projectRHS)


class PoissonEqn(_LinSys):
    """PoissonEqn(solField, rhsField, c) (src/linsys/PoissonEqn.h:3): A = c*Laplacian."""

    def __init__(self, solField: Field, rhsField: Field | None, c, opts: SolverOpts | None = None):
        self.solField, self.rhsField, self.c = solField, rhsField, float(c)
        self.opts = opts or solver_opts()
        h = _vp()
        _check(load_library().se_poisson_create(solField._h, rhsField._h if rhsField else None,
                                                self.c, ctypes.byref(self.opts),
                                                ctypes.byref(h)))
        self._h = h

    def Solve(self, removeNullSpace: bool = False, options: str = "",
              raise_on_diverge: bool = False, projectRHS: bool = False):
        """PoissonEqn::Solve(removeNullSpace) with the options prefix "poisson_";
        projectRHS as for HelmholtzEqn.Solve."""
        if options:
            o = SolverOpts.from_buffer_copy(self.opts)
            _check(_lib.se_solver_opts_parse(ctypes.byref(o), b"poisson_", options.encode()))
            self.set_opts(o)
        return self._solve(removeNullSpace, raise_on_diverge, projectRHS)


def solve_batch(systems, removeNullSpace: bool = False, raise_on_diverge: bool = False):
    """Solve several HelmholtzEqn/PoissonEqn systems in one call
    (se_linsys_solve_batch); returns one stats dict per system."""
    n = len(systems)
    arr = (_vp * n)(*[s._h for s in systems])
    st = (SolveStats * n)()
    rc = load_library().se_linsys_solve_batch(arr, n, int(bool(removeNullSpace)), st)
    if rc == SE_ERR_NOT_CONVERGED and not raise_on_diverge:
        rc = SE_OK
    _check(rc)
    out = [s.as_dict() for s in st]
    for sys_, o in zip(systems, out):
        sys_.stats = o
    return out


class Server:
    """The continuous-batching request server (se_server_*). Arrays passed to
    submit() are kept alive until wait() returns their result."""

    def __init__(self, slots: int = 8, device_gib: float = 16.0):
        h = _vp()
        rc = load_library().se_server_create(int(slots), float(device_gib), ctypes.byref(h))
        if rc:
            raise SEError(rc, "se_server_create failed")
        self._h = h
        self._keep = {}

    def submit(self, kind, nEls, N, lo, hi, periodic, field_in, aux=None, bcs=(0, 0, 0, 0),
               c=-1.0, nu=-1.0, dt=1.0, poisson=False, opts=None, steps=0, sl_dt=0.0, out=None):
        """Queue a request; `out` (optional) is a preallocated float64 result
        array (page-locked memory avoids the server's staging copies)."""
        fin = np.ascontiguousarray(field_in, dtype=np.float64)
        fa = None if aux is None else np.ascontiguousarray(aux, dtype=np.float64)
        if out is None:
            out = np.empty(len(fin))
        r = Request()
        r.kind = kind
        r.nEls[:] = [int(nEls[0]), int(nEls[1])]
        r.N = int(N)
        r.min[:] = [float(lo[0]), float(lo[1])]
        r.max[:] = [float(hi[0]), float(hi[1])]
        r.periodic[:] = [int(bool(periodic[0])), int(bool(periodic[1]))]
        r.bcs[:] = [int(bool(b)) for b in bcs]
        r.c, r.nu, r.dt, r.poisson = float(c), float(nu), float(dt), int(bool(poisson))
        r.opts = opts if opts is not None else solver_opts(rtol=1e-10, mode=MODE_EXACT,
                                                           method=METHOD_FDM)
        r.steps, r.sl_dt = int(steps), float(sl_dt)
        r.in_ = fin.ctypes.data
        r.aux = None if fa is None else fa.ctypes.data
        r.out = out.ctypes.data
        t = ctypes.c_longlong()
        rc = _lib.se_server_submit(self._h, ctypes.byref(r), ctypes.byref(t))
        if rc:
            raise SEError(rc, "se_server_submit failed")
        self._keep[t.value] = (fin, fa, out, r)
        return t.value

    def request(self, kind, nEls, N, lo, hi, periodic, field_in, aux=None, bcs=(0, 0, 0, 0),
                c=-1.0, nu=-1.0, dt=1.0, poisson=False, opts=None, steps=0, sl_dt=0.0, out=None):
        """A reusable request structure for submit_request(): the arrays are
        referenced, not copied, and must stay alive (and in place) while any
        request made from it is in flight."""
        r = Request()
        r.kind = kind
        r.nEls[:] = [int(nEls[0]), int(nEls[1])]
        r.N = int(N)
        r.min[:] = [float(lo[0]), float(lo[1])]
        r.max[:] = [float(hi[0]), float(hi[1])]
        r.periodic[:] = [int(bool(periodic[0])), int(bool(periodic[1]))]
        r.bcs[:] = [int(bool(b)) for b in bcs]
        r.c, r.nu, r.dt, r.poisson = float(c), float(nu), float(dt), int(bool(poisson))
        r.opts = opts if opts is not None else solver_opts(rtol=1e-10, mode=MODE_EXACT,
                                                           method=METHOD_FDM)
        r.steps, r.sl_dt = int(steps), float(sl_dt)
        r.in_ = field_in.ctypes.data
        r.aux = None if aux is None else aux.ctypes.data
        r.out = out.ctypes.data
        return r

    def submit_request(self, r):
        """Queue a request made by request(); returns its ticket."""
        t = ctypes.c_longlong()
        rc = _lib.se_server_submit(self._h, ctypes.byref(r), ctypes.byref(t))
        if rc:
            raise SEError(rc, "se_server_submit failed")
        return t.value

    def wait_request(self, ticket, res=None):
        """Wait for a request queued by submit_request(); returns the filled
        Result structure (res, if given, is reused)."""
        res = res if res is not None else Result()
        rc = _lib.se_server_wait(self._h, ctypes.c_longlong(ticket), ctypes.byref(res))
        if rc:
            raise SEError(rc, "se_server_wait failed")
        return res

    def wait(self, ticket):
        res = Result()
        rc = _lib.se_server_wait(self._h, ctypes.c_longlong(ticket), ctypes.byref(res))
        if rc:
            raise SEError(rc, "se_server_wait failed")
        fin, fa, out, r = self._keep.pop(ticket)
        return out, {"status": res.status, "reason": res.reason, "its": res.its,
                     "queued_ms": res.queued_ms, "latency_ms": res.latency_ms,
                     "error": res.error.decode(errors="replace")}

    def close(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.se_server_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()


class TwoLayerQGEqn:
    """TwoLayerQGEqn(psi1, omega1, psi2, omega2, F1, F2, beta, E2, r, nu,
    tau_e, dt) (src/qg/TwoLayerQGEqn.h) over se_qg2_*: Solve() advances the
    four fields one step in place (second order when the previous fields are
    given, which are then replaced by the fields before the step)."""

    def __init__(self, psi1: Field, omega1: Field, psi2: Field, omega2: Field, F1, F2, beta, E2,
                 r, nu, tau_e: Field, dt, opts: SolverOpts | None = None):
        self.fields = (psi1, omega1, psi2, omega2, tau_e)
        self.opts = opts if opts is not None else solver_opts()
        h = _vp()
        _check(load_library().se_qg2_create(psi1._h, omega1._h, psi2._h, omega2._h, float(F1),
                                            float(F2), float(beta), float(E2), float(r),
                                            float(nu), tau_e._h, float(dt),
                                            ctypes.byref(self.opts), ctypes.byref(h)))
        self._h = h

    def Solve(self, psi1Prev: Field | None = None, omega1Prev: Field | None = None,
              psi2Prev: Field | None = None, omega2Prev: Field | None = None,
              raise_on_diverge: bool = False):
        prev = (psi1Prev, omega1Prev, psi2Prev, omega2Prev)
        rc = _lib.se_qg2_solve(self._h, *[f._h if f is not None else None for f in prev])
        if rc == SE_ERR_NOT_CONVERGED and not raise_on_diverge:
            rc = SE_OK  # the step completed, as the reference's does
        _check(rc)

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.se_qg2_destroy(self._h)
            self._h = None


class NavierStokesEqn:
    """NavierStokesEqn(velocity, pressure, dt) (src/ns/NavierStokesEqn.h)
    over se_ns_*: Solve(velocity, pressure, prevVel, nu, svvCutoff) advances
    the velocity and pressure one splitting step in place (second order when
    prevVel is given; prevVel is only read). The velocity's Dirichlet sides
    are its BCs' (per-component BCs, or one scalar BCs for both components);
    ``stats`` holds the last step's pressure, u and v solver statistics."""

    def __init__(self, velocity: Field, pressure: Field, dt, opts: SolverOpts | None = None):
        b = velocity.bcs
        comps = (None, None) if b is None else (b.components or (b, b))
        self.fields, self.bcs = (velocity, pressure), comps
        self.opts = opts if opts is not None else solver_opts()
        h = _vp()
        _check(load_library().se_ns_create(velocity._h, pressure._h,
                                           comps[0]._h if comps[0] else None,
                                           comps[1]._h if comps[1] else None, float(dt),
                                           ctypes.byref(self.opts), ctypes.byref(h)))
        self._h = h
        self.stats = None

    def Solve(self, velocity: Field, pressure: Field, prevVel: Field | None, nu,
              svvCutoff: int = 0, raise_on_diverge: bool = False):
        rc = _lib.se_ns_solve(self._h, velocity._h, pressure._h,
                              prevVel._h if prevVel is not None else None, float(nu),
                              int(svvCutoff))
        if rc == SE_ERR_NOT_CONVERGED and not raise_on_diverge:
            rc = SE_OK  # the step completed, as the reference's does
        _check(rc)
        st = (SolveStats * 3)()
        _check(_lib.se_ns_stats(self._h, st))
        self.stats = [x.as_dict() for x in st]
        return self.stats

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.se_ns_destroy(self._h)
            self._h = None


def WriteXDMFHeader(timeStep: int):
    """WriteXDMFHeader (src/base/Utils.cpp:53-71): starts XDMF.<step>.xmf."""
    _check(load_library().se_write_xdmf_header(int(timeStep)))


def WriteXDMF(fields, nFields: int, timeStep: int, time: float, dt: float):
    """WriteXDMF (src/base/Utils.cpp:91-168): time.<step>.ts, each field saved
    as <name>.<step>.seb, and the grid appended to XDMF.<step>.xmf; the mesh
    file is the one Mesh.Save wrote under the first field's mesh name."""
    fs = list(fields)[:nFields]
    hs = (_vp * len(fs))(*[f._h for f in fs])
    names = (ctypes.c_char_p * len(fs))(*[f.name.encode() for f in fs])
    _check(load_library().se_write_xdmf(hs, names, len(fs), fs[0].mesh.name.encode(),
                                        int(timeStep), float(time), float(dt)))


def WriteXDMFFooter(timeStep: int):
    _check(load_library().se_write_xdmf_footer(int(timeStep)))


def WriteXDMFTemporal(nTimeSteps: int, dumpEvery: int):
    """WriteXDMFTemporal (src/base/Utils.cpp:170-229)."""
    _check(load_library().se_write_xdmf_temporal(int(nTimeSteps), int(dumpEvery)))


def GenVel(psi: Field, name: str = "vel") -> Field:
    """TwoLayerQGEqn::GenVel: a new 2-component field (-d psi/dy, d psi/dx)
    at every vertex of psi's mesh (no boundary conditions)."""
    vel = Field(name, psi.mesh, 2, None)
    _check(load_library().se_field_gen_vel(psi._h, vel._h))
    return vel


def CalcTimeStep(velocity: Field, courantNo: float) -> float:
    out = ctypes.c_double()
    _check(load_library().se_calc_time_step(velocity._h, float(courantNo), ctypes.byref(out)))
    return out.value


def FieldError(numeric: Field, analytic: Field, dof: int = 0, normalise: bool = True) -> float:
    out = ctypes.c_double()
    _check(load_library().se_field_error(numeric._h, analytic._h, dof, int(normalise),
                                         ctypes.byref(out)))
    return out.value
