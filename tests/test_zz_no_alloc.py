"""The no-allocation solve entry point (se_helmholtz_solve_noalloc).

It serves callers that cannot call cudaMalloc -- a model driver that
reserves its device-memory budget up front while other components share the
GPU, or a time loop that cannot take an allocation's implicit device-wide
synchronisation mid-step. The test calls it through the C-ABI on
caller-owned device arrays and checks its solutions against the allocating
HelmholtzEqn/PoissonEqn path (se_linsys_*) on two calls in a row, with the
solver tolerance of the other solver tests (1e-12 relative), and checks that
a system beyond its size limit is refused with a clear error.

This file is named to be collected last, so that a run stopping at the first
failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _arr(t, v):
    return (t * len(v))(*v)


def run_noalloc(S, case, rhs, sol, c, nu, dt, poisson=False, rtol=1e-12, null=False, opts=None,
                free_bytes=None, allow_diverge=False):
    lib = S.load_library()
    nx, ny, N, lo, hi, per, bc = case
    rhs_d = None if rhs is None else torch.tensor(rhs, device="cuda", dtype=torch.float64)
    sol_d = torch.tensor(sol, device="cuda", dtype=torch.float64)
    st = S.SolveStats()
    if opts is None:
        opts = S.solver_opts(rtol=rtol)
    torch.cuda.synchronize()
    if free_bytes is not None:
        free_bytes.append(torch.cuda.mem_get_info()[0])
    rc = lib.se_helmholtz_solve_noalloc(
        _arr(ctypes.c_int, [nx, ny]), N, _arr(ctypes.c_double, lo), _arr(ctypes.c_double, hi),
        _arr(ctypes.c_int, [int(per[0]), int(per[1])]), _arr(ctypes.c_int, [int(b) for b in bc]),
        c, nu, dt, int(poisson), ctypes.byref(opts), int(null),
        ctypes.c_void_p(None if rhs_d is None else rhs_d.data_ptr()),
        ctypes.c_void_p(sol_d.data_ptr()), ctypes.byref(st))
    if free_bytes is not None:
        torch.cuda.synchronize()
        free_bytes.append(torch.cuda.mem_get_info()[0])
    if rc == S.SE_ERR_NOT_CONVERGED and allow_diverge:
        rc = 0
    if rc != 0:
        raise S.SEError(rc, lib.se_last_error().decode())
    return sol_d.cpu().numpy(), st.as_dict()


def run_linsys(S, case, rhs, sol, c, nu, dt, poisson=False, rtol=1e-12, null=False):
    nx, ny, N, lo, hi, per, bc = case
    m = S.Mesh("m", [nx, ny], "legendre", N, list(lo), list(hi), list(per))
    b = S.BCs(*bc, m)
    fs, fr = S.Field("sol", m, 1, b), S.Field("rhs", m, 1, b)
    fs.vals = sol
    if rhs is not None:
        fr.vals = rhs
    opts = S.solver_opts(rtol=rtol)
    if poisson:
        ls = S.PoissonEqn(fs, fr if rhs is not None else None, c, opts)
        st = ls.Solve(removeNullSpace=bool(null), projectRHS=null == 2)
    else:
        ls = S.HelmholtzEqn(fs, fr if rhs is not None else None, c, nu, dt, 0, opts)
        st = ls.Solve("helm_", removeNullSpace=bool(null), projectRHS=null == 2)
    return fs.vals, st


def fields(case, seed):
    nx, ny, N, lo, hi, per, bc = case
    nvx, nvy = nx * N + 1, ny * N + 1
    rng = np.random.default_rng(seed)
    x = np.linspace(lo[0], hi[0], nvx)[None, :] * np.ones((nvy, 1))
    y = np.linspace(lo[1], hi[1], nvy)[:, None] * np.ones((1, nvx))
    sol = (np.sin(2 * x + 0.3) * np.cos(3 * y) + 0.05 * rng.standard_normal((nvy, nvx))).ravel()
    rhs = (np.cos(x) * np.sin(2 * y + 1) + 0.05 * rng.standard_normal((nvy, nvx))).ravel()
    if per[0]:
        sol.reshape(nvy, nvx)[:, -1] = sol.reshape(nvy, nvx)[:, 0]
        rhs.reshape(nvy, nvx)[:, -1] = rhs.reshape(nvy, nvx)[:, 0]
    if per[1]:
        sol.reshape(nvy, nvx)[-1, :] = sol.reshape(nvy, nvx)[0, :]
        rhs.reshape(nvy, nvx)[-1, :] = rhs.reshape(nvy, nvx)[0, :]
    return rhs, sol


CHANNEL = (8, 6, 6, (0.0, 0.0), (2.0, 1.0), (True, False), (True, True, False, False))
BOX = (5, 7, 4, (-1.0, -1.0), (1.0, 1.0), (False, False), (True, True, True, True))


def test_noalloc_matches_linsys_two_calls_in_a_row(segpu):
    # first call: a periodic channel with Dirichlet walls (Helmholtz)
    rhs, sol = fields(CHANNEL, 1)
    got1, st1 = run_noalloc(segpu, CHANNEL, rhs, sol, -3.0, -1.0, 1.0)
    ref1, rs1 = run_linsys(segpu, CHANNEL, rhs, sol, -3.0, -1.0, 1.0)
    assert st1["reason"] == rs1["reason"] == 2 and st1["its"] == rs1["its"]
    assert np.abs(got1 - ref1).max() <= TOL * np.abs(ref1).max()
    # second call, right after: another mesh and operator (Poisson, all
    # Dirichlet), so the scratch left by the first call is overwritten
    rhs, sol = fields(BOX, 2)
    got2, st2 = run_noalloc(segpu, BOX, rhs, sol, -1.0, 0.0, 0.0, poisson=True)
    ref2, rs2 = run_linsys(segpu, BOX, rhs, sol, -1.0, 0.0, 0.0, poisson=True)
    assert st2["reason"] == rs2["reason"] == 2 and st2["its"] == rs2["its"]
    assert np.abs(got2 - ref2).max() <= TOL * np.abs(ref2).max()
    # and the first system once more: same answer as the first call
    rhs, sol = fields(CHANNEL, 1)
    got3, st3 = run_noalloc(segpu, CHANNEL, rhs, sol, -3.0, -1.0, 1.0)
    assert np.abs(got3 - got1).max() <= TOL * np.abs(ref1).max()
    assert st3["its"] == st1["its"]


def test_noalloc_refuses_systems_beyond_its_limit(segpu):
    big = (40, 40, 8, (0.0, 0.0), (1.0, 1.0), (True, True), (False, False, False, False))
    nvx = 40 * 8 + 1
    with pytest.raises(segpu.SEError) as e:
        run_noalloc(segpu, big, None, np.zeros(nvx * nvx), -1.0, -1.0, 1.0)
    assert e.value.code == segpu.SE_ERR_UNSUPPORTED
    assert "no-allocation limit" in str(e.value)


def test_noalloc_allocates_no_device_memory(segpu):
    # after a first call (which looks the static array up), a call leaves the
    # device's free memory exactly as it found it
    rhs, sol = fields(CHANNEL, 3)
    run_noalloc(segpu, CHANNEL, rhs, sol, -3.0, -1.0, 1.0)
    free = []
    run_noalloc(segpu, CHANNEL, rhs, sol, -3.0, -1.0, 1.0, free_bytes=free)
    assert free[0] == free[1]


PERIODIC = (6, 6, 5, (0.0, 0.0), (1.0, 1.0), (True, True), (False, False, False, False))


def test_noalloc_periodic_poisson_null_space(segpu):
    # a singular periodic Poisson system with the constant null space removed
    # (mode 1: projected from every preconditioned residual; mode 2: the
    # right-hand side projected onto the range first), against the allocating
    # path: same reason, same iteration count, same solution when converged
    rhs, sol = fields(PERIODIC, 4)
    for null in (1, 2):
        got, st = run_noalloc(segpu, PERIODIC, rhs, sol, -1.0, 0.0, 0.0, poisson=True,
                              rtol=1e-10, null=null, allow_diverge=True)
        ref, rs = run_linsys(segpu, PERIODIC, rhs, sol, -1.0, 0.0, 0.0, poisson=True,
                             rtol=1e-10, null=null)
        assert st["reason"] == rs["reason"] and st["its"] == rs["its"]
        if rs["reason"] > 0:
            assert np.abs(got - ref).max() <= TOL * np.abs(ref).max()


def test_noalloc_refuses_other_methods_and_precisions(segpu):
    rhs, sol = fields(CHANNEL, 5)
    for kw in ({"method": segpu.METHOD_FDM}, {"precision": segpu.PREC_MIXED},
               {"precision": segpu.PREC_BF16}):
        opts = segpu.solver_opts(rtol=1e-10, **kw)
        with pytest.raises(segpu.SEError) as e:
            run_noalloc(segpu, CHANNEL, rhs, sol, -3.0, -1.0, 1.0, opts=opts)
        assert e.value.code == segpu.SE_ERR_UNSUPPORTED
    # an unknown norm type is an argument error, as in se_helmholtz_create
    opts = segpu.solver_opts(rtol=1e-10)
    opts.norm_type = 7
    with pytest.raises(segpu.SEError) as e:
        run_noalloc(segpu, CHANNEL, rhs, sol, -3.0, -1.0, 1.0, opts=opts)
    assert e.value.code == segpu.SE_ERR_ARG
