"""The two-layer QG step (TwoLayerQGEqn, src/qg/TwoLayerQGEqn.cpp) on the GPU
through the C-ABI (se_qg2_*), against the oracle's restatement of the same
step (oracle.QG2), on a channel: periodic in x, walls (Dirichlet) in y.

One first-order step, then two second-order steps with the previous fields.
Both sides solve the inversions to rtol 1e-12 (CG drop-in, and FDM on the
GPU side) with the true-Jacobian Laplacian, and advect with accurate
cardinal functions, so the fields agree to 1e-9 of their magnitude (the
inversions' tolerance amplified through the step)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-9
NX, NY, N = 12, 6, 5
LO, HI = (0.0, 0.0), (2.0, 1.0)
PARAMS = dict(F1=25.0, F2=25.0, beta=0.5, E2=0.02, r=0.01, nu=1e-4, dt=0.005)


def initial(X):
    x, y = X[:, 0], X[:, 1]
    psi1 = 0.1 * np.cos(np.pi * y) + 0.01 * np.sin(np.pi * x) * np.sin(np.pi * y)
    psi2 = -0.05 * np.cos(np.pi * y) + 0.005 * np.cos(np.pi * x) * np.sin(2 * np.pi * y)
    om1 = -0.1 * np.pi ** 2 * np.cos(np.pi * y) + 0.03 * np.sin(np.pi * x) * np.cos(np.pi * y)
    om2 = 0.05 * np.pi ** 2 * np.cos(np.pi * y) - 0.02 * np.cos(np.pi * x) * np.sin(np.pi * y)
    tau_e = 0.02 * np.cos(np.pi * y)
    return psi1, om1, psi2, om2, tau_e


def rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


@pytest.mark.parametrize("method", ["cg", "fdm"])
def test_qg_steps_match_oracle(segpu, oracle, method):
    om = oracle.Mesh(NX, NY, N, LO, HI, (True, False), accurate=True)
    X = om.verts()
    psi1, om1, psi2, om2, tau_e = [om.periodic_update(v) for v in initial(X)]
    bcs = (True, True, False, False)
    ref = oracle.QG2(om, bcs, psi1, om1, psi2, om2, tau_e=tau_e, rtol=1e-12, **PARAMS)

    m = segpu.Mesh("m", [NX, NY], "legendre", N, list(LO), list(HI), [True, False])
    bc = segpu.BCs(*bcs, m)
    fields = [segpu.Field(name, m, 1, bc if name.startswith("psi") else None)
              for name in ("psi1", "omega1", "psi2", "omega2", "tau_e")]
    for f, v in zip(fields, (psi1, om1, psi2, om2, tau_e)):
        f.vals = v
    prev = [segpu.Field(f"{name}-prev", m, 1, None) for name in ("psi1", "omega1", "psi2", "omega2")]
    for f, v in zip(prev, (psi1, om1, psi2, om2)):
        f.vals = v
    opts = segpu.solver_opts(rtol=1e-12, mode=segpu.MODE_EXACT,
                             method=segpu.METHOD_FDM if method == "fdm" else segpu.METHOD_CG)
    qg = segpu.TwoLayerQGEqn(*fields[:4], PARAMS["F1"], PARAMS["F2"], PARAMS["beta"],
                             PARAMS["E2"], PARAMS["r"], PARAMS["nu"], fields[4], PARAMS["dt"],
                             opts)

    qg.Solve()  # first order
    ref.step(None)
    saved = (psi1, om1, psi2, om2)
    for k in range(2):  # second order; prev fields hold the fields before the step
        qg.Solve(*prev)
        saved = ref.step(saved)
        for f, v in zip(prev, saved):
            assert rel(f.vals, v) < TOL
    for f, v in zip(fields[:4], (ref.psi1, ref.omega1, ref.psi2, ref.omega2)):
        assert np.all(np.isfinite(f.vals))
        assert rel(f.vals, v) < TOL
    # the step changed the fields (not a no-op)
    assert rel(fields[0].vals, psi1) > 1e-6


def test_qg_rejects_mismatched_fields(segpu):
    m = segpu.Mesh("m", [4, 4], "legendre", 4, [0, 0], [1, 1], [True, False])
    bc = segpu.BCs(True, True, False, False, m)
    fs = [segpu.Field("f", m, 1, bc) for _ in range(5)]
    vel = segpu.Field("v", m, 2, None)
    with pytest.raises(segpu.SEError):
        segpu.TwoLayerQGEqn(fs[0], vel, fs[2], fs[3], 1, 1, 0, 0, 0, 0, fs[4], 0.01)
    nobc = segpu.Field("p", m, 1, None)
    with pytest.raises(segpu.SEError):
        segpu.TwoLayerQGEqn(nobc, fs[1], fs[2], fs[3], 1, 1, 0, 0, 0, 0, fs[4], 0.01)
