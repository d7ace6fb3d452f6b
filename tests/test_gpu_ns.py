"""The Navier-Stokes splitting step (NavierStokesEqn, src/ns/NavierStokesEqn.cpp)
on the GPU through the C-ABI (se_ns_*), against the oracle's restatement of
the same step (oracle.NS).

The Taylor vortex of the reference's own model (models/taylor-vortex/
TaylorVortex.cpp: the box [-pi/2, pi/2]^2, u Dirichlet on the left and right
sides and v on the bottom and top, a separate pressure mesh of the same
geometry with no Dirichlet sides) and a channel periodic in x with v
Dirichlet on the walls. One first-order step, then two second-order steps
with the previous velocity. Both sides solve the pressure and viscous systems
(CG drop-in, and FDM on the GPU side) with the true-Jacobian Laplacian and
advect with accurate cardinal functions, so the velocity and pressure agree
to 1000 times the solver tolerance relative to their magnitude (rtol 1e-12;
the pressure operator's condition number, about 2.4e3 here, turns a
residual of rtol into a solution error up to that size).
The pressure right-hand side (the vertex divergence, mass weighted) is off
the Neumann operator's range by a few 1e-6 of its size; on it the plain
Jacobi CG with the null space projected out stagnates (near 1e-7 in the
Taylor vortex's second-order step) and ends on an indefinite inner product.
Both sides therefore solve the consistent system that iteration approaches
(the right-hand side minus its component along the diagonal), where CG and
FDM converge."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HALF_PI = 0.5 * np.pi


def taylor(X, t, nu):
    x, y = X[:, 0], X[:, 1]
    u = np.stack([-np.cos(x) * np.sin(y), np.sin(x) * np.cos(y)], 1) * np.exp(-2 * nu * t)
    p = -0.25 * (np.cos(2 * x) + np.cos(2 * y)) * np.exp(-4 * nu * t)
    return u, p


def channel(X, t, nu):
    x, y = X[:, 0], X[:, 1]
    u = np.stack([0.3 * np.cos(np.pi * y) + 0.05 * np.sin(np.pi * x) * np.cos(np.pi * y),
                  0.05 * np.cos(np.pi * x) * np.sin(np.pi * y)], 1)
    p = 0.01 * np.cos(np.pi * x) * np.cos(np.pi * y)
    return u, p


CASES = {
    # name: (nEls, N, lo, hi, periodic, bcs_u, bcs_v (bottom, top, left, right), initial, nu,
    #        rtol)
    "taylor": (6, 5, (-HALF_PI, -HALF_PI), (HALF_PI, HALF_PI), (False, False),
               (False, False, True, True), (True, True, False, False), taylor, 1.0, 1e-12),
    "channel": (6, 6, (0.0, -1.0), (2.0, 1.0), (True, False),
                (False, False, False, False), (True, True, False, False), channel, 0.01, 1e-12),
}


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def setup(segpu, oracle, name, method, mode):
    ne, N, lo, hi, per, bu, bv, init, nu, rtol = CASES[name]
    om = oracle.Mesh(ne, ne, N, lo, hi, per, accurate=True)
    X = om.verts()
    dx = (hi[0] - lo[0]) / ne / 8
    dt = min(0.5 * (hi[0] - lo[0]) / (2.0 * ne), 0.5 * dx * dx / nu)
    prev, _ = init(X, 0.0, nu)
    vel, pres = init(X, dt, nu)
    prev = np.stack([om.periodic_update(prev[:, d]) for d in range(2)], 1)
    vel = np.stack([om.periodic_update(vel[:, d]) for d in range(2)], 1)
    pres = om.periodic_update(pres)
    ref = oracle.NS(om, bu, bv, dt, quirk=(mode == segpu.MODE_REFERENCE), rtol=rtol)

    vm = segpu.Mesh("vMesh", [ne, ne], "legendre", N, list(lo), list(hi), list(per))
    pm = segpu.Mesh("pMesh", [ne, ne], "legendre", N, list(lo), list(hi), list(per))
    vbcs = segpu.BCs([bu[0], bv[0]], [bu[1], bv[1]], [bu[2], bv[2]], [bu[3], bv[3]], vm)
    pbcs = segpu.BCs(False, False, False, False, pm)
    velocity = segpu.Field("velocity", vm, 2, vbcs)
    prevVel = segpu.Field("prevVel", vm, 2, vbcs)
    pressure = segpu.Field("pressure", pm, 1, pbcs)
    velocity.vals, prevVel.vals, pressure.vals = vel, prev, pres
    opts = segpu.solver_opts(rtol=rtol, mode=mode,
                             method=segpu.METHOD_FDM if method == "fdm" else segpu.METHOD_CG)
    ns = segpu.NavierStokesEqn(velocity, pressure, dt, opts)
    return dict(ref=ref, ns=ns, velocity=velocity, prevVel=prevVel, pressure=pressure,
                vel=vel, prev=prev, pres=pres, nu=nu, dt=dt, X=X, init=init, tol=1000 * rtol,
                om=om)


@pytest.mark.parametrize("name", ["taylor", "channel"])
@pytest.mark.parametrize("method", ["cg", "fdm"])
def test_ns_steps_match_oracle(segpu, oracle, name, method):
    c = setup(segpu, oracle, name, method, segpu.MODE_EXACT)
    ns, ref, nu, TOL = c["ns"], c["ref"], c["nu"], c["tol"]
    velocity, pressure, prevVel = c["velocity"], c["pressure"], c["prevVel"]
    # first order (NavierStokesEqn::SolveFirstOrder)
    st = ns.Solve(velocity, pressure, None, nu, 0, raise_on_diverge=True)
    assert all(s["reason"] > 0 for s in st)
    vel, pres, _ = ref.step(c["vel"], c["pres"], None, nu)
    assert rel(velocity.vals, vel) < TOL
    assert rel(pressure.vals, pres) < TOL
    # second order with the previous velocity, as the reference's models drive it
    for _ in range(2):
        saved = velocity.vals
        st = ns.Solve(velocity, pressure, prevVel, nu, 0, raise_on_diverge=True)
        assert all(s["reason"] > 0 for s in st)
        vel_new, pres, _ = ref.step(vel, pres, prevVel.vals, nu)
        prevVel.vals = saved
        vel = vel_new
        got = velocity.vals
        assert np.all(np.isfinite(got))
        assert rel(got, vel) < TOL
        assert rel(pressure.vals, pres) < TOL
    assert rel(velocity.vals, c["vel"]) > 1e-7  # the step changed the velocity


def test_ns_first_order_taylor_vortex_accuracy(segpu, oracle):
    """One first-order step of the decaying Taylor vortex stays within 1e-4 of
    the analytic velocity (the scheme, not only the parity)."""
    c = setup(segpu, oracle, "taylor", "fdm", segpu.MODE_EXACT)
    c["ns"].Solve(c["velocity"], c["pressure"], None, c["nu"], 0)
    ua, _ = taylor(c["X"], 2 * c["dt"], c["nu"])
    assert np.abs(c["velocity"].vals - ua).max() < 1e-4


@pytest.mark.parametrize("method", ["cg", "fdm"])
def test_ns_svv_matches_oracle(segpu, oracle, method):
    """The step with the SVV operator in the viscous systems (svvCutoff =
    N/2, as the reference's cavity-flow and Kelvin-Helmholtz models pass);
    the viscous systems are solved by CG with either method, the pressure by
    the chosen one."""
    c = setup(segpu, oracle, "channel", method, segpu.MODE_EXACT)
    ns, ref, nu, TOL = c["ns"], c["ref"], c["nu"], c["tol"]
    svv = CASES["channel"][1] // 2
    # seeded noise gives the velocity the high modes the filter acts on
    noise = 0.02 * np.random.default_rng(7).standard_normal(c["vel"].shape)
    c["vel"] = np.stack([c["om"].periodic_update(c["vel"][:, d] + noise[:, d])
                         for d in range(2)], 1)
    c["velocity"].vals = c["vel"]
    st = ns.Solve(c["velocity"], c["pressure"], None, nu, svv, raise_on_diverge=True)
    assert all(s["reason"] > 0 for s in st)
    vel, pres, _ = ref.step(c["vel"], c["pres"], None, nu, svv_cutoff=svv)
    assert rel(c["velocity"].vals, vel) < TOL
    assert rel(c["pressure"].vals, pres) < TOL
    ns.Solve(c["velocity"], c["pressure"], c["prevVel"], nu, svv, raise_on_diverge=True)
    vel2, pres2, _ = ref.step(vel, pres, c["prevVel"].vals, nu, svv_cutoff=svv)
    assert rel(c["velocity"].vals, vel2) < TOL
    assert rel(c["pressure"].vals, pres2) < TOL
    # SVV changes the result (the filter acts on this field)
    vel_plain, _, _ = ref.step(c["vel"], c["pres"], None, nu)
    assert rel(vel, vel_plain) > 1e-6


def test_ns_reference_laplacian_mode(segpu, oracle):
    """The reference's Laplacian (detJ dropped) through the whole step."""
    c = setup(segpu, oracle, "channel", "cg", segpu.MODE_REFERENCE)
    c["ns"].Solve(c["velocity"], c["pressure"], None, c["nu"], 0)
    vel, pres, _ = c["ref"].step(c["vel"], c["pres"], None, c["nu"])
    assert rel(c["velocity"].vals, vel) < c["tol"]
    assert rel(c["pressure"].vals, pres) < c["tol"]


def test_ns_rejections(segpu):
    m = segpu.Mesh("m", [4, 4], "legendre", 4, [0, 0], [1, 1], [False, False])
    other = segpu.Mesh("o", [4, 4], "legendre", 5, [0, 0], [1, 1], [False, False])
    vel = segpu.Field("v", m, 2, None)
    pres = segpu.Field("p", m, 1, None)
    with pytest.raises(segpu.SEError):
        segpu.NavierStokesEqn(pres, pres, 0.01)  # velocity needs 2 components
    with pytest.raises(segpu.SEError):
        segpu.NavierStokesEqn(vel, segpu.Field("q", other, 1, None), 0.01)  # pressure geometry
    ns = segpu.NavierStokesEqn(vel, pres, 0.01)
    with pytest.raises(segpu.SEError):
        ns.Solve(vel, pres, None, 1.0, 5)  # svvCutoff above N = 4
    with pytest.raises(segpu.SEError):
        ns.Solve(segpu.Field("w", m, 2, None), pres, None, 1.0, 0)  # not the system's field
    with pytest.raises(segpu.SEError):
        ns.Solve(vel, pres, pres, 1.0, 0)  # previous velocity with 1 component
