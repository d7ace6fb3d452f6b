"""GPU parity of the matrix-free Helmholtz/Poisson operator and the
persistent Jacobi-PCG (src/linsys/HelmholtzEqn.cpp, PoissonEqn.cpp) against
the oracle's assembled AIJ operator and restated PETSc KSPCG, through the
C-ABI.

Tolerances (FP64): operator apply within 2e-11 of the |A||x| row scale --
the reference builds every element matrix through a numerically computed
Jacobian, so its own element matrices differ from element to element by up
to 5.1e-12 relative on these cases (identical in exact arithmetic on SE's
uniform meshes);
solutions of rtol=1e-12 solves within 1e-8 relative; iteration counts within
2 of the oracle's; repeated solves bit-identical.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

CASES = [
    # (nx, ny, N, lo, hi, periodic, bcs(bottom, top, left, right))
    (5, 4, 4, (0.0, 0.0), (1.0, 1.0), (True, True), (False, False, False, False)),
    (6, 3, 6, (0.0, 0.0), (2.0, 1.0), (True, False), (True, True, False, False)),
    (4, 5, 5, (-1.0, -1.0), (1.0, 1.0), (False, False), (True, True, True, True)),
    (3, 4, 3, (-1.0, 0.0), (1.0, 1.5), (False, False), (True, False, True, False)),
    (4, 3, 8, (0.0, 0.0), (1.0, 2.0), (True, False), (False, True, False, False)),
    (3, 3, 7, (0.0, 0.0), (1.0, 1.0), (False, False), (False, False, False, False)),
]


# Order-8 meshes large enough for tiles that the apply stages with TMA:
# periodic interior tiles; a Dirichlet left end (staged columns shifted by
# one to keep the copy 16-byte aligned) with natural right and bottom ends
# (zero fill); an odd number of unknowns per row (ordinary loads only).
CASES8 = [
    (26, 14, 8, (0.0, 0.0), (1.0, 1.0), (True, True), (False, False, False, False)),
    (25, 13, 8, (0.0, 0.0), (2.0, 1.0), (False, False), (False, True, True, False)),
    (24, 15, 8, (-1.0, 0.0), (1.0, 1.0), (False, False), (False, False, False, False)),
    (20, 17, 8, (0.0, 0.0), (1.0, 1.0), (True, False), (True, True, False, False)),
]

# Order-4 to order-7 meshes of several element-factored tiles (64 x 16,
# 60 x 20, 60 x 24 and 63 x 28 vertices) with partial tiles at the far ends:
# doubly periodic, channels, Dirichlet ends, natural ends everywhere.
CASES_EF = [
    (37, 9, 4, (0.0, 0.0), (1.0, 1.0), (True, True), (False, False, False, False)),
    (35, 10, 4, (0.0, 0.0), (2.0, 1.0), (False, False), (False, True, True, False)),
    (23, 11, 6, (0.0, 0.0), (1.0, 1.0), (True, True), (False, False, False, False)),
    (21, 9, 6, (0.0, 0.0), (1.0, 1.0), (True, False), (True, True, False, False)),
    (22, 7, 6, (-1.0, 0.0), (1.0, 1.0), (False, False), (False, False, False, False)),
    (27, 9, 5, (0.0, 0.0), (1.0, 1.0), (True, True), (False, False, False, False)),
    (25, 10, 5, (0.0, 0.0), (1.0, 1.0), (False, False), (True, False, False, True)),
    (20, 9, 7, (0.0, 0.0), (1.0, 1.0), (True, True), (False, False, False, False)),
    (19, 8, 7, (0.0, 0.0), (2.0, 1.0), (True, False), (True, True, False, False)),
]


def build(S, O, case, c, nu, dt, quirk, poisson=False, seed=0):
    nx, ny, N, lo, hi, per, bc = case
    om = O.Mesh(nx, ny, N, lo, hi, per)
    X = om.verts()
    rng = np.random.default_rng(seed)
    sol = np.sin(3 * X[:, 0] + 1) * np.cos(2 * X[:, 1]) + 0.1 * rng.standard_normal(om.nv)
    rhs = np.cos(2 * X[:, 0]) * np.sin(X[:, 1] + 0.5) + 0.1 * rng.standard_normal(om.nv)
    sol, rhs = om.periodic_update(sol), om.periodic_update(rhs)
    m = S.Mesh("m", [nx, ny], "legendre", N, list(lo), list(hi), list(per))
    b = S.BCs(*bc, m)
    fs, fr = S.Field("sol", m, 1, b), S.Field("rhs", m, 1, b)
    fs.vals, fr.vals = sol, rhs
    opts = S.solver_opts(rtol=1e-12, mode=S.MODE_REFERENCE if quirk else S.MODE_EXACT)
    ls = S.PoissonEqn(fs, fr, c, opts) if poisson else S.HelmholtzEqn(fs, fr, c, nu, dt, 0, opts)
    f2v, v2f = om.bcs_maps(*bc)
    if poisson:
        A = O.CSR(om, f2v, len(v2f), 0.0, c, quirk, sol)
    else:
        A = O.CSR(om, f2v, len(v2f), c, nu * dt, quirk, sol)
    return om, m, fs, fr, ls, A, f2v, v2f, sol, rhs


@pytest.mark.parametrize("case", range(len(CASES)))
@pytest.mark.parametrize("quirk", [True, False])
def test_apply_matches_assembled_operator(segpu, oracle, case, quirk):
    om, m, fs, fr, ls, A, f2v, v2f, sol, rhs = build(segpu, oracle, CASES[case], -2.0, -1.0, 0.5,
                                                     quirk)
    n = ls.vecSize
    assert n == len(v2f)
    x = np.random.default_rng(case).standard_normal(n)
    ref = A.matvec(x)
    xd = torch.tensor(x, device="cuda", dtype=torch.float64)
    yd = torch.zeros(n, device="cuda", dtype=torch.float64)
    ls.apply(xd.data_ptr(), yd.data_ptr())
    torch.cuda.synchronize()
    rowptr, col, val, _ = A.arrays()
    scale = np.array([np.abs(val[rowptr[i]:rowptr[i + 1]]).sum() for i in range(n)]) * np.abs(x).max()
    assert (np.abs(yd.cpu().numpy() - ref) / scale).max() < 2e-11
    d = torch.zeros(n, device="cuda", dtype=torch.float64)
    ls.diagonal(d.data_ptr())
    torch.cuda.synchronize()
    diag = np.array([val[rowptr[i]:rowptr[i + 1]][col[rowptr[i]:rowptr[i + 1]] == i][0] for i in range(n)])
    assert np.abs(d.cpu().numpy() - diag).max() <= 2e-11 * np.abs(diag).max()


@pytest.mark.parametrize("case", [("o8", k) for k in range(len(CASES8))]
                         + [("ef", k) for k in range(len(CASES_EF))])
def test_apply_factored_tiles(segpu, oracle, case):
    """The element-factored FP64 apply (orders 4 to 8) over meshes of several
    tiles, against the oracle's assembled CSR operator."""
    spec = (CASES8 if case[0] == "o8" else CASES_EF)[case[1]]
    case = case[1] + (0 if case[0] == "o8" else 10)
    om, m, fs, fr, ls, A, f2v, v2f, sol, rhs = build(segpu, oracle, spec, -2.0, -1.0, 0.5, False)
    n = ls.vecSize
    x = np.random.default_rng(100 + case).standard_normal(n)
    ref = A.matvec(x)
    xd = torch.tensor(x, device="cuda", dtype=torch.float64)
    yd = torch.full((n,), float("nan"), device="cuda", dtype=torch.float64)
    for _ in range(2):  # the second call reuses the per-device launch set-up
        ls.apply(xd.data_ptr(), yd.data_ptr())
        torch.cuda.synchronize()
        rowptr, col, val, _ = A.arrays()
        scale = np.array([np.abs(val[rowptr[i]:rowptr[i + 1]]).sum() for i in range(n)]) * np.abs(x).max()
        assert (np.abs(yd.cpu().numpy() - ref) / scale).max() < 2e-11


@pytest.mark.parametrize("case", list(range(len(CASES))) + ["o8-" + str(k) for k in range(len(CASES8))])
@pytest.mark.parametrize("prec", ["bf16", "fp16"])
def test_low_precision_apply(segpu, oracle, case, prec):
    """se_linsys_apply_low: x rounded to BF16/FP16, operator and arithmetic in
    FP32. Against the oracle's FP64 CSR on the same rounded x, the error is
    bounded by FP32 rounding of the coefficients and the sums: 1e-6 of the
    row's absolute sum times max|x|."""
    spec = CASES8[int(case[3:])] if isinstance(case, str) else CASES[case]
    om, m, fs, fr, ls, A, f2v, v2f, sol, rhs = build(segpu, oracle, spec, -2.0, -1.0, 0.5, False)
    n = ls.vecSize
    dt = torch.bfloat16 if prec == "bf16" else torch.float16
    x = torch.tensor(np.random.default_rng(10 + len(str(case))).standard_normal(n), dtype=dt)
    ref = A.matvec(x.double().numpy())
    xd = x.cuda()
    yd = torch.zeros(n, device="cuda", dtype=torch.float32)
    ls.apply_low(xd.data_ptr(), yd.data_ptr(), segpu.PREC_BF16 if prec == "bf16" else segpu.PREC_FP16)
    torch.cuda.synchronize()
    rowptr, col, val, _ = A.arrays()
    scale = np.array([np.abs(val[rowptr[i]:rowptr[i + 1]]).sum() for i in range(n)]) * float(x.abs().max())
    assert (np.abs(yd.cpu().double().numpy() - ref) / scale).max() < 1e-6


@pytest.mark.parametrize("case", [0, 1, 4])
def test_fdm_apply_inverts_operator(segpu, oracle, case):
    """se_linsys_fdm_apply: A (A^{-1} r) = r to FP64 rounding (relative to
    |A| |x|), Helmholtz operators on periodic and Dirichlet meshes."""
    om, m, fs, fr, ls, A, f2v, v2f, sol, rhs = build(segpu, oracle, CASES[case], -2.0, -1.0, 0.5,
                                                     False)
    n = ls.vecSize
    r = np.random.default_rng(7 + case).standard_normal(n)
    rd = torch.tensor(r, device="cuda", dtype=torch.float64)
    xd = torch.zeros(n, device="cuda", dtype=torch.float64)
    ls.fdm_apply(rd.data_ptr(), xd.data_ptr())
    torch.cuda.synchronize()
    x = xd.cpu().numpy()
    rowptr, col, val, _ = A.arrays()
    scale = np.array([np.abs(val[rowptr[i]:rowptr[i + 1]]).sum() for i in range(n)]) * np.abs(x).max()
    assert (np.abs(A.matvec(x) - r) / scale).max() < 1e-12


# Doubly periodic meshes with 2^k elements per direction: the FP64 inverse
# takes the Bloch form (an FFT across elements and p x p blocks per
# wavenumber) instead of dense eigenvector products.
CASES_BLOCH = [
    (8, 16, 4, (0.0, 0.0), (1.0, 2.0), (True, True), (False, False, False, False)),
    (16, 4, 6, (0.0, 0.0), (2.0, 1.0), (True, True), (False, False, False, False)),
    (32, 32, 8, (0.0, 0.0), (1.0, 1.0), (True, True), (False, False, False, False)),
    (2, 8, 12, (-1.0, 0.0), (1.0, 1.0), (True, True), (False, False, False, False)),
]


@pytest.mark.parametrize("case", CASES_BLOCH)
@pytest.mark.parametrize("quirk", [False, True])
def test_fdm_bloch_inverts_operator(segpu, oracle, case, quirk):
    """The Bloch-form inverse: A (A^{-1} r) = r to FP64 rounding (relative to
    |A| |x|: 1e-12, 3e-12 at order 12, whose element blocks span a wider
    range of eigenvalues), for the true-Jacobian and the detJ = 1 operators,
    square and stretched elements, orders 4 to 12."""
    om, m, fs, fr, ls, A, f2v, v2f, sol, rhs = build(segpu, oracle, case, -2.0, -1.0, 0.5, quirk)
    n = ls.vecSize
    r = np.random.default_rng(11).standard_normal(n)
    rd = torch.tensor(r, device="cuda", dtype=torch.float64)
    xd = torch.zeros(n, device="cuda", dtype=torch.float64)
    ls.fdm_apply(rd.data_ptr(), xd.data_ptr())
    torch.cuda.synchronize()
    x = xd.cpu().numpy()
    rowptr, col, val, _ = A.arrays()
    scale = np.array([np.abs(val[rowptr[i]:rowptr[i + 1]]).sum() for i in range(n)]) * np.abs(x).max()
    assert (np.abs(A.matvec(x) - r) / scale).max() < (3e-12 if case[2] == 12 else 1e-12)


@pytest.mark.parametrize("case", CASES_BLOCH)
def test_fdm_bloch_solve_matches_oracle(segpu, oracle, case):
    """FDM solve in Bloch form, refined in FP64 to rtol 1e-10: the oracle's CG
    solution at rtol 1e-14 within 1e-8 of its magnitude; a periodic Poisson
    system with its null space removed likewise."""
    om, m, fs, fr, ls, A, f2v, v2f, sol, rhs = build(segpu, oracle, case, -3.0, -1.0, 1.0, False,
                                                     seed=21)
    ref_sol, st = oracle.helmholtz_solve(om, sol, rhs, -3.0, -1.0, 1.0, bcs=case[6], quirk=False,
                                         rtol=1e-14)
    ls.set_opts(segpu.solver_opts(rtol=1e-10, method=segpu.METHOD_FDM, mode=segpu.MODE_EXACT))
    out = ls.Solve("helm_")
    assert out["reason"] == 2 and out["its"] <= 2, out
    assert np.abs(fs.vals - ref_sol).max() <= 1e-8 * np.abs(ref_sol).max()
    # Poisson, constant null space
    X = om.verts()
    f = om.periodic_update(np.cos(2 * np.pi * X[:, 0] / (case[4][0] - case[3][0]))
                           * np.sin(2 * np.pi * X[:, 1] / (case[4][1] - case[3][1])))
    bc = segpu.BCs(False, False, False, False, m)
    u, rf = segpu.Field("u", m, 1, bc), segpu.Field("f", m, 1, bc)
    rf.vals = f
    ps = segpu.PoissonEqn(u, rf, 1.0, segpu.solver_opts(rtol=1e-10, method=segpu.METHOD_FDM,
                                                        mode=segpu.MODE_EXACT))
    out = ps.Solve(removeNullSpace=True)
    assert out["reason"] == 2, out
    u_cg = segpu.Field("ucg", m, 1, bc)
    pc = segpu.PoissonEqn(u_cg, rf, 1.0, segpu.solver_opts(rtol=1e-13, mode=segpu.MODE_EXACT))
    pc.Solve(removeNullSpace=True)
    ref = u_cg.vals - u_cg.vals.mean()
    got = u.vals - u.vals.mean()
    assert np.abs(got - ref).max() <= 1e-8 * np.abs(ref).max()


@pytest.mark.parametrize("case", [0, 1, 4])
def test_fdm_apply_tensor_cores_inverts_operator(segpu, oracle, case):
    """se_linsys_fdm_apply_prec(SE_PREC_MIXED): the FDM inverse on the tcgen05
    tensor cores (TF32 hi/lo operand pairs, three products per K step, FP32
    accumulation) inverts the operator to about 1e-6 of |A| |x|, and agrees
    with the FP64 inverse to 2e-5 of its magnitude."""
    om, m, fs, fr, ls, A, f2v, v2f, sol, rhs = build(segpu, oracle, CASES[case], -2.0, -1.0, 0.5,
                                                     False)
    n = ls.vecSize
    r = np.random.default_rng(11 + case).standard_normal(n)
    rd = torch.tensor(r, device="cuda", dtype=torch.float64)
    xt = torch.zeros(n, device="cuda", dtype=torch.float64)
    x64 = torch.zeros(n, device="cuda", dtype=torch.float64)
    ls.fdm_apply(rd.data_ptr(), xt.data_ptr(), segpu.PREC_MIXED)
    ls.fdm_apply(rd.data_ptr(), x64.data_ptr())
    torch.cuda.synchronize()
    x, xr = xt.cpu().numpy(), x64.cpu().numpy()
    rowptr, col, val, _ = A.arrays()
    scale = np.array([np.abs(val[rowptr[i]:rowptr[i + 1]]).sum() for i in range(n)]) * np.abs(x).max()
    assert (np.abs(A.matvec(x) - r) / scale).max() < 1e-5
    assert np.abs(x - xr).max() <= 2e-5 * np.abs(xr).max()
    # twice in a row on the same buffers: the same result (deterministic)
    xt2 = torch.zeros(n, device="cuda", dtype=torch.float64)
    ls.fdm_apply(rd.data_ptr(), xt2.data_ptr(), segpu.PREC_MIXED)
    assert torch.equal(xt, xt2)


def test_option_checks(segpu):
    m = segpu.Mesh("m", [4, 4], "legendre", 4, [0, 0], [1, 1], [True, True])
    b = segpu.BCs(False, False, False, False, m)
    u, r = segpu.Field("u", m, 1, b), segpu.Field("r", m, 1, b)
    for bad in (dict(precision=segpu.PREC_FP16, method=segpu.METHOD_FDM),
                dict(precision=segpu.PREC_MIXED, method=segpu.METHOD_CG),
                dict(precision=segpu.PREC_FP64_TC, method=segpu.METHOD_CG),
                dict(method=7), dict(norm_type=5)):
        with pytest.raises(segpu.SEError):
            segpu.HelmholtzEqn(u, r, -1.0, -1.0, 1.0, 0, segpu.solver_opts(**bad))


@pytest.mark.parametrize("case", range(len(CASES)))
def test_helmholtz_solve_matches_oracle(segpu, oracle, case):
    om, m, fs, fr, ls, A, f2v, v2f, sol, rhs = build(segpu, oracle, CASES[case], -3.0, -1.0, 1.0,
                                                     True, seed=case + 10)
    ref_sol, st = oracle.helmholtz_solve(om, sol, rhs, -3.0, -1.0, 1.0, bcs=CASES[case][6],
                                         quirk=True, rtol=1e-12)
    out = ls.Solve("helm_")
    assert st["reason"] == 2 and out["reason"] == 2
    assert abs(out["its"] - st["its"]) <= 2, (out, st)
    got = fs.vals
    assert np.abs(got - ref_sol).max() <= 1e-8 * np.abs(ref_sol).max()
    # Dirichlet values untouched, periodic copies refreshed
    assert np.array_equal(got[f2v < 0], sol[f2v < 0])


def test_solve_deterministic_and_reusable(segpu, oracle):
    om, m, fs, fr, ls, A, *_ = build(segpu, oracle, CASES[1], -1.0, -1.0, 1.0, True)
    a = ls.Solve("helm_")
    v1 = fs.vals
    b = ls.Solve("helm_")
    v2 = fs.vals
    a.pop("kernel_ms"), b.pop("kernel_ms")
    assert a == b and np.array_equal(v1, v2)


def test_config0_exact_modal_solution(segpu, oracle):
    """(lap - 1) u = f on the doubly periodic 16x16, p=6 unit square, f a
    seeded sum of 8 Fourier modes; CG + Jacobi to rtol 1e-10 in the exact
    (true Jacobian) mode reaches the modal solution to the discretisation
    error, with the oracle's iteration count."""
    rng = np.random.default_rng(0)
    m = segpu.Mesh("m", [16, 16], "legendre", 6, [0, 0], [1, 1], [True, True])
    X = m.verts
    f, u = np.zeros(len(X)), np.zeros(len(X))
    for _ in range(8):
        kx, ky = rng.integers(1, 7, size=2)
        a, b = rng.standard_normal(2)
        ph = 2 * np.pi * (kx * X[:, 0] + ky * X[:, 1])
        mode = a * np.cos(ph) + b * np.sin(ph)
        f += mode
        u += mode / (-(4 * np.pi ** 2 * (kx * kx + ky * ky)) - 1.0)
    bc = segpu.BCs(False, False, False, False, m)
    fs, fr = segpu.Field("u", m, 1, bc), segpu.Field("f", m, 1, bc)
    fr.vals = f
    ls = segpu.HelmholtzEqn(fs, fr, -1.0, -1.0, 1.0, 0,
                            segpu.solver_opts(rtol=1e-10, mode=segpu.MODE_EXACT))
    st = ls.Solve("helm_")
    om = oracle.Mesh(16, 16, 6)
    _, ost = oracle.helmholtz_solve(om, np.zeros(om.nv), f, -1.0, -1.0, 1.0, quirk=False,
                                    rtol=1e-10)
    assert st["reason"] == 2 and abs(st["its"] - ost["its"]) <= 2
    got = fs.vals
    assert np.linalg.norm(got - u) / np.linalg.norm(u) < 1e-7
    ua = segpu.Field("ua", m, 1, bc)
    ua.vals = u
    assert segpu.FieldError(fs, ua) < 1e-7


def test_poisson_null_space(segpu, oracle):
    """Doubly periodic Poisson with a constant null space removed, for a
    consistent right-hand side (zero mean): converges like the oracle. With an
    inconsistent one (nonzero mean) the projected Jacobi-CG breaks down and
    both report KSP_DIVERGED_INDEFINITE_PC at the same iteration; with the
    right-hand side projected onto the range (mode 2) CG and FDM converge to
    the oracle's solution of the consistent system."""
    case = (6, 6, 5, (0.0, 0.0), (1.0, 1.0), (True, True), (False, False, False, False))
    om, m, fs, fr, ls, A, f2v, v2f, sol, rhs = build(segpu, oracle, case, -1.0, 0, 0, True,
                                                     poisson=True)
    X = om.verts()
    rhs = om.periodic_update(np.sin(2 * np.pi * X[:, 0]) * np.cos(4 * np.pi * X[:, 1])
                             + np.cos(2 * np.pi * X[:, 1]))
    fr.vals = rhs
    ref_sol, st = oracle.helmholtz_solve(om, sol, rhs, -1.0, 0, 0, quirk=True, rtol=1e-10,
                                         remove_null_space=True, poisson=True)
    out = ls.Solve(removeNullSpace=True)
    assert out["reason"] == st["reason"] == 2
    assert abs(out["its"] - st["its"]) <= 2
    got = fs.vals
    assert np.abs(got - ref_sol).max() <= 1e-7 * np.abs(ref_sol).max()
    bad = om.periodic_update(rhs + 0.3)
    fr.vals = bad
    _, st2 = oracle.helmholtz_solve(om, sol, bad, -1.0, 0, 0, quirk=True, rtol=1e-10,
                                    remove_null_space=True, poisson=True)
    out2 = ls.Solve(removeNullSpace=True)
    assert st2["reason"] == out2["reason"] == -8
    assert abs(st2["its"] - out2["its"]) <= 1
    # mode 2: the right-hand side projected onto the range first; CG and FDM
    # both converge to the oracle's solution of that consistent system
    ref3, st3 = oracle.helmholtz_solve(om, sol, bad, -1.0, 0, 0, quirk=True, rtol=1e-12,
                                       remove_null_space=True, poisson=True, project_rhs=True)
    assert st3["reason"] == 2
    for method in (segpu.METHOD_CG, segpu.METHOD_FDM):
        ls.set_opts(segpu.solver_opts(rtol=1e-12, method=method))
        out3 = ls.Solve(removeNullSpace=True, projectRHS=True, raise_on_diverge=True)
        assert out3["reason"] == 2
        assert np.abs(fs.vals - ref3).max() <= 1e-9 * np.abs(ref3).max()
    assert segpu.load_library().se_linsys_solve(ls._h, 3, None) == segpu.SE_ERR_ARG


@pytest.mark.parametrize("case", [CASES_BLOCH[0], CASES[1]], ids=["bloch", "dense-channel"])
@pytest.mark.parametrize("prec", ["PREC_FP64", "PREC_FP64_TC"])
def test_fdm_first_step_keeps_initial_decision(segpu, oracle, case, prec):
    """FP64 first refinement steps run outside the refinement loop (the
    Bloch form and the dense inverse; FP64 and FP64-then-tensor-core). When
    the initial test has already decided, that step adds nothing. With
    max_it = 0 the FDM solve ends as the CG drop-in does: reason -3 (ITS) at
    iteration 0, the same field (zero initial guess, Dirichlet values kept).
    A zero right-hand side with zero boundary values converges at iteration
    0 with a zero solution. The next solve of the same system converges to
    the oracle's solution as before."""
    om, m, fs, fr, ls, *_ = build(segpu, oracle, case, -3.0, -1.0, 1.0, False, seed=5)
    sol0, rhs = fs.vals.copy(), fr.vals.copy()
    fdm = dict(rtol=1e-10, method=segpu.METHOD_FDM, precision=getattr(segpu, prec),
               mode=segpu.MODE_EXACT)
    fields = []
    for opts in (dict(fdm, max_it=0), dict(rtol=1e-10, max_it=0, mode=segpu.MODE_EXACT)):
        fs.vals = sol0
        ls.set_opts(segpu.solver_opts(**opts))
        ls.Assemble()
        st = ls.Solve("helm_")
        assert st["reason"] == -3 and st["its"] == 0, (opts, st)
        fields.append(fs.vals.copy())
    assert np.array_equal(fields[0], fields[1])
    fs.vals, fr.vals = 0.0, 0.0
    ls.set_opts(segpu.solver_opts(**fdm))
    ls.Assemble()
    st = ls.Solve("helm_")
    assert st["its"] == 0 and st["reason"] in (2, 3), st
    assert np.abs(fs.vals).max() == 0.0
    fs.vals, fr.vals = sol0, rhs
    ls.Assemble()
    st = ls.Solve("helm_")
    assert st["reason"] == 2 and st["its"] <= 4, st
    ref_sol, _ = oracle.helmholtz_solve(om, sol0, rhs, -3.0, -1.0, 1.0, bcs=case[6], quirk=False,
                                        rtol=1e-14)
    assert np.abs(fs.vals - ref_sol).max() <= 1e-8 * np.abs(ref_sol).max()


def test_solver_reasons(segpu, oracle):
    om, m, fs, fr, ls, *_ = build(segpu, oracle, CASES[0], -1.0, -1.0, 1.0, True)
    ls.set_opts(segpu.solver_opts(rtol=1e-14, max_it=3))
    st = ls.Solve("helm_")
    assert st["reason"] == -3 and st["its"] == 3
    with pytest.raises(segpu.SEError) as e:
        ls.Solve("helm_", raise_on_diverge=True)
    assert e.value.code == segpu.SE_ERR_NOT_CONVERGED
    # zero right-hand side converges at iteration 0
    fr.vals = 0.0
    ls.set_opts(segpu.solver_opts(rtol=1e-10))
    st = ls.Solve("helm_")
    assert st["its"] == 0 and st["reason"] in (2, 3)
    with pytest.raises(segpu.SEError) as e:
        segpu.HelmholtzEqn(fs, fr, 1.0, 1.0, 1.0, 5)  # svvCutoff above N = 4
    assert e.value.code == segpu.SE_ERR_ARG


def test_field_error_calc_time_step(segpu, oracle):
    om = oracle.Mesh(5, 4, 6, (0, 0), (2, 1), (True, False))
    X = om.verts()
    a = np.sin(X[:, 0]) + X[:, 1] ** 2
    b = a + 1e-3 * np.cos(5 * X[:, 0])
    m = segpu.Mesh("m", [5, 4], "legendre", 6, [0, 0], [2, 1], [True, False])
    fa, fb = segpu.Field("a", m, 1, None), segpu.Field("b", m, 1, None)
    fa.vals, fb.vals = a, b
    ref = om.field_error(b, a)
    assert abs(segpu.FieldError(fb, fa) - ref) <= 1e-10 * ref
    v = np.stack([np.sin(X[:, 0]), np.cos(3 * X[:, 1])], 1)
    fv = segpu.Field("v", m, 2, None)
    fv.vals = v
    assert abs(segpu.CalcTimeStep(fv, 2.0) - om.calc_time_step(v, 2.0)) <= 1e-15


# ------------------------------------------------- fast diagonalization ----
@pytest.mark.parametrize("case", range(len(CASES)))
@pytest.mark.parametrize("prec", [0, 1, 2, 4])
def test_fdm_solve_matches_oracle(segpu, oracle, case, prec):
    """FDM (exact 1-D eigenvector transforms) refined in FP64 to rtol 1e-10 in
    the true preconditioned residual reaches the oracle's CG solution of the
    same system (run to rtol 1e-14), for FP64 transforms, TF32 hi/lo
    products on the tcgen05 tensor cores, BF16, and FP64 for the first step
    with tensor-core steps after."""
    om, m, fs, fr, ls, A, f2v, v2f, sol, rhs = build(segpu, oracle, CASES[case], -3.0, -1.0, 1.0,
                                                     True, seed=case + 20)
    ref_sol, st = oracle.helmholtz_solve(om, sol, rhs, -3.0, -1.0, 1.0, bcs=CASES[case][6],
                                         quirk=True, rtol=1e-14)
    ls.set_opts(segpu.solver_opts(rtol=1e-10, method=segpu.METHOD_FDM, precision=prec,
                                  max_it=40))
    out = ls.Solve("helm_")
    assert out["reason"] == 2, out
    if prec == 0:
        assert out["its"] <= 2
    if prec == 4:  # at most one FP64 step more than needed
        assert out["its"] <= 3
    got = fs.vals
    assert np.abs(got - ref_sol).max() <= 1e-8 * np.abs(ref_sol).max()
    assert np.array_equal(got[f2v < 0], sol[f2v < 0])


@pytest.mark.parametrize("case", [CASES_EF[0], CASES_EF[1], CASES_EF[3], CASES_EF[6], CASES_EF[8],
                                  CASES8[0], CASES8[1]])
@pytest.mark.parametrize("prec", ["bf16", "fp16"])
def test_cg_reduced_precision_apply_refined(segpu, oracle, case, prec):
    """CG whose operator apply reads its direction vector in BF16 / FP16 and
    computes in FP32, inside FP64 iterative refinement with the double-double
    residual, to rtol 1e-10 (the Laplacian with its true Jacobian: the
    reference's detJ = 1 form on these stretched elements has condition
    numbers beyond BF16's reach): the oracle's CG solution at rtol 1e-14
    within 1e-8 of its magnitude, reached over several refinement steps;
    Dirichlet values untouched."""
    om, m, fs, fr, ls, A, f2v, v2f, sol, rhs = build(segpu, oracle, case, -3.0, -1.0, 1.0, False,
                                                     seed=7)
    ref_sol, st = oracle.helmholtz_solve(om, sol, rhs, -3.0, -1.0, 1.0, bcs=case[6], quirk=False,
                                         rtol=1e-14)
    p = segpu.PREC_BF16 if prec == "bf16" else segpu.PREC_FP16
    ls.set_opts(segpu.solver_opts(rtol=1e-10, method=segpu.METHOD_CG, precision=p,
                                  mode=segpu.MODE_EXACT, max_it=100000))
    out = ls.Solve("helm_")
    assert out["reason"] == 2, out
    assert out["outer_its"] >= 2 and out["rnorm"] <= 1e-10 * out["rnorm0"], out
    got = fs.vals
    assert np.abs(got - ref_sol).max() <= 1e-8 * np.abs(ref_sol).max()
    assert np.array_equal(got[f2v < 0], sol[f2v < 0])
    # deterministic: the same solve again gives the same bits
    again = ls.Solve("helm_")
    assert again["its"] == out["its"] and np.array_equal(fs.vals, got)


def test_cg_reduced_precision_stall_reported(segpu, oracle):
    """Where BF16's rounding times the condition number is past 1 (the detJ = 1
    Laplacian on elements stretched 4:1, nearly singular against the mass
    term), the refinement stops gaining and the solve says so
    (SE_KSP_DIVERGED_BREAKDOWN) instead of running to max_it or reporting
    convergence."""
    om, m, fs, fr, ls, A, f2v, v2f, sol, rhs = build(segpu, oracle, CASES_EF[0], -3.0, -1.0, 1.0,
                                                     True, seed=7)
    ls.set_opts(segpu.solver_opts(rtol=1e-10, method=segpu.METHOD_CG, precision=segpu.PREC_BF16,
                                  max_it=1000000))
    out = ls.Solve("helm_")
    assert out["reason"] in (2, -5), out
    if out["reason"] == 2:
        assert out["rnorm"] <= 1e-10 * out["rnorm0"]


def test_cg_reduced_precision_refusals(segpu):
    """The reduced-precision CG covers orders 4-8 without SVV or null-space
    removal; the rest is refused, not run in another precision."""
    o = segpu.solver_opts(rtol=1e-10, method=segpu.METHOD_CG, precision=segpu.PREC_BF16)
    m = segpu.Mesh("m", [4, 4], "legendre", 3, [0, 0], [1, 1], [True, True])
    b = segpu.BCs(False, False, False, False, m)
    u, r = segpu.Field("u", m, 1, b), segpu.Field("r", m, 1, b)
    r.vals = np.cos(2 * np.pi * m.verts[:, 0])
    with pytest.raises(segpu.SEError) as e:
        segpu.HelmholtzEqn(u, r, -1.0, -1.0, 1.0, 0, o).Solve("helm_")
    assert e.value.code == segpu.SE_ERR_UNSUPPORTED
    m6 = segpu.Mesh("m6", [4, 4], "legendre", 6, [0, 0], [1, 1], [True, True])
    b6 = segpu.BCs(False, False, False, False, m6)
    u6, r6 = segpu.Field("u", m6, 1, b6), segpu.Field("r", m6, 1, b6)
    r6.vals = np.cos(2 * np.pi * m6.verts[:, 0])
    with pytest.raises(segpu.SEError) as e:
        segpu.PoissonEqn(u6, r6, 1.0, o).Solve(removeNullSpace=True)
    assert e.value.code == segpu.SE_ERR_UNSUPPORTED


def test_fdm_config0_exact_modal_and_null_space(segpu, oracle):
    rng = np.random.default_rng(0)
    m = segpu.Mesh("m", [16, 16], "legendre", 6, [0, 0], [1, 1], [True, True])
    X = m.verts
    f, u = np.zeros(len(X)), np.zeros(len(X))
    for _ in range(8):
        kx, ky = rng.integers(1, 7, size=2)
        a, b = rng.standard_normal(2)
        ph = 2 * np.pi * (kx * X[:, 0] + ky * X[:, 1])
        mode = a * np.cos(ph) + b * np.sin(ph)
        f += mode
        u += mode / (-(4 * np.pi ** 2 * (kx * kx + ky * ky)) - 1.0)
    bc = segpu.BCs(False, False, False, False, m)
    fs, fr = segpu.Field("u", m, 1, bc), segpu.Field("f", m, 1, bc)
    fr.vals = f
    for prec in (0, 2):
        ls = segpu.HelmholtzEqn(fs, fr, -1.0, -1.0, 1.0, 0,
                                segpu.solver_opts(rtol=1e-10, mode=segpu.MODE_EXACT,
                                                  method=segpu.METHOD_FDM, precision=prec))
        st = ls.Solve("helm_")
        assert st["reason"] == 2
        assert np.linalg.norm(fs.vals - u) / np.linalg.norm(u) < 1e-7
    # periodic Poisson with the constant null space: matches the oracle CG
    om = oracle.Mesh(16, 16, 6)
    g = om.periodic_update(np.sin(2 * np.pi * X[:, 0]) * np.cos(4 * np.pi * X[:, 1]))
    fr.vals = g
    ref, st = oracle.helmholtz_solve(om, np.zeros(om.nv), g, -1.0, 0, 0, quirk=True, rtol=1e-13,
                                     remove_null_space=True, poisson=True)
    ps = segpu.PoissonEqn(fs, fr, -1.0, segpu.solver_opts(rtol=1e-10, method=segpu.METHOD_FDM))
    out = ps.Solve(removeNullSpace=True)
    assert out["reason"] == 2
    assert np.abs(fs.vals - ref).max() <= 1e-8 * np.abs(ref).max()


def test_fdm_options_string(segpu):
    o = segpu.solver_opts("helm_", "-helm_ksp_type preonly -helm_pc_type fdm -helm_ksp_rtol 1e-9")
    assert o.method == segpu.METHOD_FDM and o.rtol == 1e-9


def test_async_solve_and_download(segpu, oracle):
    """se_linsys_solve_async/finish report the solve's own statistics (the
    state copy has reached the host when finish returns), and
    se_field_download_async matches the synchronous download after a
    synchronize."""
    import ctypes
    om, m, fs, fr, ls, *_ = build(segpu, oracle, CASES[1], -1.0, -1.0, 1.0, False)
    ls.set_opts(segpu.solver_opts(rtol=1e-12, mode=segpu.MODE_EXACT, method=segpu.METHOD_FDM))
    ref = ls.Solve("helm_")
    want = fs.vals
    assert ref["reason"] == 2 and ref["its"] >= 1
    for k in range(3):
        ls.solve_async()
        st = ls.solve_finish()
        assert (st["reason"], st["its"]) == (ref["reason"], ref["its"])
        assert st["rnorm0"] == ref["rnorm0"]
    ls.set_opts(segpu.solver_opts(rtol=1e-6, mode=segpu.MODE_EXACT, method=segpu.METHOD_FDM))
    ls.solve_async()
    assert ls.solve_finish()["its"] <= ref["its"]
    out = torch.full((len(want),), float("nan"), dtype=torch.float64).pin_memory()
    ptr = ctypes.cast(out.data_ptr(), ctypes.POINTER(ctypes.c_double))
    assert segpu.load_library().se_field_download_async(fs._h, ptr) == 0
    segpu.synchronize()
    assert np.array_equal(out.numpy(), fs.vals)


@pytest.mark.parametrize("case", [0, 1, 2, 4])
def test_residual_double_double(segpu, oracle, case):
    """se_linsys_residual: r = b - A x with the sums in double-double equals
    the oracle's CSR residual to 2e-11 of |A| |x| + |b| (the apply's parity
    bound: the assembled CSR and the Kronecker form round their coefficients
    differently), with the element-factored kernel at orders 4 to 8 and the
    general one otherwise; and when b is the library's own apply of x the
    residual is only that apply's rounding (the cancellation keeps its
    digits)."""
    om, m, fs, fr, ls, A, f2v, v2f, sol, rhs = build(segpu, oracle, CASES[case], -2.0, -1.0, 0.5,
                                                     False)
    n = ls.vecSize
    rng = np.random.default_rng(31 + case)
    x = rng.standard_normal(n)
    b = rng.standard_normal(n)
    xd = torch.tensor(x, device="cuda", dtype=torch.float64)
    bd = torch.tensor(b, device="cuda", dtype=torch.float64)
    rd = torch.empty_like(xd)
    ls.residual(xd.data_ptr(), bd.data_ptr(), rd.data_ptr())
    torch.cuda.synchronize()
    rowptr, col, val, _ = A.arrays()
    absA = np.array([np.abs(val[rowptr[i]:rowptr[i + 1]]).sum() for i in range(n)])
    ref = b - A.matvec(x)
    assert (np.abs(rd.cpu().numpy() - ref) / (absA * np.abs(x).max() + np.abs(b))).max() < 2e-11
    # b = the library's own FP64 apply of x: the residual is that apply's
    # rounding, a few units of |A| |x| in the last place, not more
    bd2 = torch.empty_like(xd)
    ls.apply(xd.data_ptr(), bd2.data_ptr())
    ls.residual(xd.data_ptr(), bd2.data_ptr(), rd.data_ptr())
    torch.cuda.synchronize()
    assert np.abs(rd.cpu().numpy()).max() <= 1e-13 * (absA * np.abs(x).max()).max()
