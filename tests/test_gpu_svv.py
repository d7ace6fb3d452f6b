"""HelmholtzEqn with the spectral vanishing viscosity operator (svvCutoff != 0:
src/linsys/HelmholtzEqn.cpp:71, src/base/SVV.cpp) on the GPU through the
C-ABI, against the oracle's assembled operator built from the literal SVV
element matrices (themselves pinned to the reference's own
SVV::AssembleElement in test_oracle_svv.py).

The GPU applies the term in its factored form 2 dt detJ (T kron S) inside the
CG kernel's staged apply (the element blocks reach the halo's corners) and in
the Dirichlet lifting. Tolerances as for the operator without SVV: the apply
within 2e-11 of the |A||x| row scale, rtol=1e-12 solutions within 1e-8
relative with iteration counts within 2 of the oracle's."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

CASES = [
    # (nx, ny, N, lo, hi, periodic, bcs(bottom, top, left, right), svvCutoff)
    (5, 4, 4, (0.0, 0.0), (1.0, 1.0), (True, True), (False, False, False, False), 2),
    (6, 3, 6, (0.0, 0.0), (2.0, 1.0), (True, False), (True, True, False, False), 3),
    (4, 5, 5, (-1.0, -1.0), (1.0, 1.0), (False, False), (True, True, True, True), 2),
    (3, 4, 8, (-1.0, 0.0), (1.0, 1.5), (False, False), (True, False, True, False), 4),
    (4, 3, 7, (0.0, 0.0), (1.0, 2.0), (True, False), (False, True, False, False), 3),
    (3, 3, 8, (0.0, 0.0), (1.0, 1.0), (False, False), (False, False, False, False), 6),
]
C, NU, DT = 1.5, 0.2, 0.05


def build(S, O, case, quirk, seed=0):
    nx, ny, N, lo, hi, per, bc, svv = case
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
    ls = S.HelmholtzEqn(fs, fr, C, NU, DT, svv, opts)
    f2v, v2f = om.bcs_maps(*bc)
    A = O.CSR(om, f2v, len(v2f), C, NU * DT, quirk, sol, svv=(DT, svv))
    return om, m, fs, fr, ls, A, f2v, v2f, sol, rhs


@pytest.mark.parametrize("case", range(len(CASES)))
@pytest.mark.parametrize("quirk", [True, False])
def test_svv_apply_and_diagonal(segpu, oracle, case, quirk):
    om, m, fs, fr, ls, A, f2v, v2f, sol, rhs = build(segpu, oracle, CASES[case], quirk)
    n = ls.vecSize
    x = np.random.default_rng(case).standard_normal(n)
    ref = A.matvec(x)
    xd = torch.tensor(x, device="cuda", dtype=torch.float64)
    yd = torch.full((n,), float("nan"), device="cuda", dtype=torch.float64)
    ls.apply(xd.data_ptr(), yd.data_ptr())
    torch.cuda.synchronize()
    rowptr, col, val, _ = A.arrays()
    scale = np.array([np.abs(val[rowptr[i]:rowptr[i + 1]]).sum() for i in range(n)]) * np.abs(x).max()
    assert (np.abs(yd.cpu().numpy() - ref) / scale).max() < 2e-11
    d = torch.zeros(n, device="cuda", dtype=torch.float64)
    ls.diagonal(d.data_ptr())
    torch.cuda.synchronize()
    diag = np.array([val[rowptr[i]:rowptr[i + 1]][col[rowptr[i]:rowptr[i + 1]] == i][0]
                     for i in range(n)])
    assert np.abs(d.cpu().numpy() - diag).max() <= 2e-11 * np.abs(diag).max()
    # the SVV term is really there: the operator without it differs
    A0 = oracle.CSR(om, f2v, len(v2f), C, NU * DT, quirk, sol)
    assert np.abs(A0.matvec(x) - ref).max() > 1e-6 * np.abs(ref).max()


@pytest.mark.parametrize("case", range(len(CASES)))
def test_svv_solve_matches_oracle(segpu, oracle, case):
    om, m, fs, fr, ls, A, f2v, v2f, sol, rhs = build(segpu, oracle, CASES[case], True,
                                                     seed=case + 3)
    ref_sol, st = oracle.helmholtz_solve(om, sol, rhs, C, NU, DT, bcs=CASES[case][6], quirk=True,
                                         rtol=1e-12, svv_cutoff=CASES[case][7])
    out = ls.Solve("helm_")
    assert st["reason"] == 2 and out["reason"] == 2
    assert abs(out["its"] - st["its"]) <= 2, (out, st)
    got = fs.vals
    assert np.abs(got - ref_sol).max() <= 1e-8 * np.abs(ref_sol).max()
    assert np.array_equal(got[f2v < 0], sol[f2v < 0])  # Dirichlet values untouched


def test_svv_refusals(segpu, oracle):
    om, m, fs, fr, ls, *_ = build(segpu, oracle, CASES[0], True)
    with pytest.raises(segpu.SEError):
        ls.set_opts(segpu.solver_opts(method=segpu.METHOD_FDM))
    with pytest.raises(segpu.SEError):
        segpu.HelmholtzEqn(fs, fr, C, NU, DT, 2, segpu.solver_opts(method=segpu.METHOD_FDM))
    with pytest.raises(segpu.SEError):
        segpu.HelmholtzEqn(fs, fr, C, NU, DT, 5)  # cutoff above N = 4
    n = ls.vecSize
    x = torch.zeros(n, device="cuda", dtype=torch.float64)
    y = torch.zeros(n, device="cuda", dtype=torch.float64)
    with pytest.raises(segpu.SEError):
        ls.fdm_apply(x.data_ptr(), y.data_ptr())
    xb = torch.zeros(n, device="cuda", dtype=torch.bfloat16)
    yf = torch.zeros(n, device="cuda", dtype=torch.float32)
    with pytest.raises(segpu.SEError):
        ls.apply_low(xb.data_ptr(), yf.data_ptr())
    # svvCutoff == N filters nothing: the same operator as without SVV
    ls_n = segpu.HelmholtzEqn(fs, fr, C, NU, DT, 4)
    ls_0 = segpu.HelmholtzEqn(fs, fr, C, NU, DT, 0)
    xr = torch.tensor(np.random.default_rng(5).standard_normal(n), device="cuda")
    yn, y0 = torch.zeros_like(xr), torch.zeros_like(xr)
    ls_n.apply(xr.data_ptr(), yn.data_ptr())
    ls_0.apply(xr.data_ptr(), y0.data_ptr())
    torch.cuda.synchronize()
    assert torch.allclose(yn, y0, rtol=1e-14, atol=1e-14 * float(y0.abs().max()))
