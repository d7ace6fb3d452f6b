"""Batched ensemble solves (se_linsys_solve_batch) against the same systems
solved one at a time.

CG systems of one polynomial order run in one persistent launch whose dot
products are segmented differently from a single solve's, so solutions agree
to 1e-10 relative and iteration counts to within 2; FDM systems run the same
graphs as single solves on other streams and agree bit for bit.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def make_systems(S, rng, count, method, p_choices=(4, 6, 8)):
    out = []
    for k in range(count):
        nx, ny = int(rng.integers(3, 12)), int(rng.integers(3, 12))
        p = int(rng.choice(p_choices))
        per = [bool(k % 3 != 2), False]
        bc = (False, False, False, False) if per[0] else (True, True, True, True)
        if per[0] and k % 2:
            bc = (True, True, False, False)
        else:
            per[1] = per[0]
        lam = float(10 ** rng.uniform(-2, 2))
        m = S.Mesh("m", [nx, ny], "legendre", p, [0.0, 0.0], [1.0, 1.5], per)
        b = S.BCs(*bc, m)
        X = m.verts
        rhs = np.sin(3 * X[:, 0] + k) * np.cos(2 * X[:, 1]) + 0.3 * np.cos(5 * X[:, 0] * X[:, 1])
        sol = 0.1 * np.cos(X[:, 0] + X[:, 1])
        if per[0]:
            nvx = m.nVerts[0]
            rhs.reshape(-1, nvx)[:, -1] = rhs.reshape(-1, nvx)[:, 0]
            sol.reshape(-1, nvx)[:, -1] = sol.reshape(-1, nvx)[:, 0]
        if per[1]:
            nvx = m.nVerts[0]
            rhs.reshape(-1, nvx)[-1, :] = rhs.reshape(-1, nvx)[0, :]
            sol.reshape(-1, nvx)[-1, :] = sol.reshape(-1, nvx)[0, :]
        fs, fr = S.Field("u", m, 1, b), S.Field("f", m, 1, b)
        fs.vals, fr.vals = sol, rhs
        ls = S.HelmholtzEqn(fs, fr, -lam, -1.0, 1.0, 0,
                            S.solver_opts(rtol=1e-11, mode=S.MODE_EXACT, method=method))
        out.append((m, b, fs, fr, ls, sol))
    return out


def test_cg_batch_matches_single_solves(segpu):
    rng = np.random.default_rng(5)
    systems = make_systems(segpu, rng, 12, segpu.METHOD_CG)
    singles = []
    for (m, b, fs, fr, ls, sol) in systems:
        st = ls.Solve("helm_")
        singles.append((fs.vals.copy(), st))
        fs.vals = sol
    stats = segpu.solve_batch([s[4] for s in systems])
    for (m, b, fs, fr, ls, sol), (ref, rst), st in zip(systems, singles, stats):
        assert st["reason"] == rst["reason"] == 2
        assert abs(st["its"] - rst["its"]) <= 2
        got = fs.vals
        assert np.abs(got - ref).max() <= 1e-10 * np.abs(ref).max()


def test_fdm_batch_bit_identical_to_single_solves(segpu):
    rng = np.random.default_rng(6)
    systems = make_systems(segpu, rng, 20, segpu.METHOD_FDM)
    singles = []
    for (m, b, fs, fr, ls, sol) in systems:
        st = ls.Solve("helm_")
        singles.append((fs.vals.copy(), st))
        fs.vals = sol
    stats = segpu.solve_batch([s[4] for s in systems])
    for (m, b, fs, fr, ls, sol), (ref, rst), st in zip(systems, singles, stats):
        assert st["reason"] == rst["reason"] == 2 and st["its"] == rst["its"]
        assert np.array_equal(fs.vals, ref)


def test_mixed_batch_and_repeat(segpu):
    rng = np.random.default_rng(7)
    systems = make_systems(segpu, rng, 6, segpu.METHOD_CG, p_choices=(6,)) + \
        make_systems(segpu, rng, 6, segpu.METHOD_FDM)
    a = segpu.solve_batch([s[4] for s in systems])
    va = [s[2].vals.copy() for s in systems]
    for s in systems:
        s[2].vals = s[5]
    b = segpu.solve_batch([s[4] for s in systems])
    for x, y, sa, sb in zip(va, [s[2].vals for s in systems], a, b):
        assert sa["reason"] == 2 and sb["reason"] == 2
        assert np.array_equal(x, y)  # deterministic, autotuned shape reused
