"""GPU parity of semi-Lagrangian advection (src/base/Advector.cpp) against
the oracle, through the C-ABI.

Two oracles check every case:
 * the oracle restatement with the reference's own cardinal-function formula
   (bit-exact with the reference), and
 * the same oracle with extended-precision Lagrange-product cardinals
   (``accurate=True``: same element search, local coordinates and 1e-8 snap).

The reference evaluates P_N'(x) as a monomial sum with pow(), which cancels
near the GLL nodes outside the snap radius: its own values there are off by
up to ~1e-16*C/|x - x_k| relative (3.6e-9 at the worst of the fixed cases
below). The GPU evaluates the cardinals in product form, accurate to
rounding. Tolerances (relative to the field's max magnitude):
  ACC_TOL = 1e-12 against the accurate oracle,
  REF_TOL = 1e-8 against the reference formula (its own error level);
departure elements bit-exact against both; element search and local
coordinates bit-exact for the same coordinates.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ACC_TOL = 1e-12
REF_TOL = 1e-8


def taylor_green(X, amp=1.0):
    x, y = X[:, 0], X[:, 1]
    return np.stack([-amp * np.sin(np.pi * x) ** 2 * np.sin(2 * np.pi * y),
                     amp * np.sin(np.pi * y) ** 2 * np.sin(2 * np.pi * x)], 1)


def make(S, nx, ny, N, lo=(0.0, 0.0), hi=(1.0, 1.0), per=(True, True)):
    return S.Mesh("m", [nx, ny], "legendre", N, list(lo), list(hi), list(per))


def rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def test_global_to_local_bit_exact(segpu, oracle, golden):
    g = golden["mesh"]
    for tag in ("pp", "px", "nn"):
        p = g[f"{tag}_params"]
        m = segpu.Mesh("m", [int(p[0]), int(p[1])], "legendre", int(p[2]), [p[3], p[4]],
                       [p[5], p[6]], [bool(p[7]), bool(p[8])])
        el, lc = m.GlobalToLocal(g[f"{tag}_pts"])
        assert np.array_equal(el, g[f"{tag}_el"])
        assert np.array_equal(lc, g[f"{tag}_lc"])


def test_interp_global_matches_reference_fixture(segpu, oracle, golden):
    g = golden["mesh"]
    for tag in ("pp", "px", "nn"):
        p = g[f"{tag}_params"]
        m = segpu.Mesh("m", [int(p[0]), int(p[1])], "legendre", int(p[2]), [p[3], p[4]],
                       [p[5], p[6]], [bool(p[7]), bool(p[8])])
        f = segpu.Field("f", m, 1, None)
        f.vals = g[f"{tag}_field"]
        pts = g[f"{tag}_pts"]
        out = f.InterpGlobal(pts)[:, 0]
        assert rel(out, g[f"{tag}_interp"][:, 0]) < REF_TOL
        om = oracle.Mesh(int(p[0]), int(p[1]), int(p[2]), (p[3], p[4]), (p[5], p[6]),
                         (bool(p[7]), bool(p[8])), accurate=True)
        assert rel(out, om.interp_global(g[f"{tag}_field"], pts)[:, 0]) < ACC_TOL
        v = segpu.Field("v", m, 2, None)
        v.vals = g[f"{tag}_vel"]
        vo = v.InterpGlobal(pts)
        assert rel(vo, g[f"{tag}_interp_vel"]) < REF_TOL
        assert rel(vo, om.interp_global(g[f"{tag}_vel"], pts, ndofs=2)) < ACC_TOL


def test_first_order_matches_reference_fixture(segpu, oracle, golden):
    s = golden["sl"]
    nx, ny, N, dt = s["first_params"]
    m = make(segpu, int(nx), int(ny), int(N))
    f, v = segpu.Field("phi", m, 1, None), segpu.Field("vel", m, 2, None)
    f.vals, v.vals = s["first_field"], s["first_vel"]
    adv = segpu.Advector(f, v)
    adv.record_departures()
    adv.Advect(dt)
    out = adv.fieldSL.vals
    assert rel(out, s["first_out"]) < REF_TOL
    om = oracle.Mesh(int(nx), int(ny), int(N), accurate=True)
    assert rel(out, om.advect(s["first_field"], s["first_vel"], dt)) < ACC_TOL
    el, xy = adv.departures()
    assert np.array_equal(el, s["first_depel"])
    assert np.abs(xy - s["first_dep"]).max() < 1e-12
    dep_acc, el_acc = om.departure_first(s["first_vel"], dt)
    assert np.array_equal(el, el_acc)
    assert np.abs(xy - dep_acc).max() < 1e-14
    # two-component field (velocity self-advection, as the NS splitting does)
    adv2 = segpu.Advector(v, v)
    adv2.Advect(dt)
    out2 = adv2.fieldSL.vals
    assert rel(out2, s["first_vel_out"]) < REF_TOL
    assert rel(out2, om.advect(s["first_vel"], s["first_vel"], dt)) < ACC_TOL


def test_second_order_matches_reference_fixture(segpu, oracle, golden):
    s = golden["sl"]
    nx, ny, N, dt = s["second_params"]
    m = make(segpu, int(nx), int(ny), int(N), hi=(2.0, 1.0), per=(True, False))
    f, fp = segpu.Field("psi", m, 1, None), segpu.Field("psiPrev", m, 1, None)
    v, vp = segpu.Field("vel", m, 2, None), segpu.Field("velPrev", m, 2, None)
    f.vals, fp.vals = s["second_field"], s["second_field_prev"]
    v.vals, vp.vals = s["second_vel"], s["second_vel_prev"]
    adv = segpu.Advector(f, v, fp, vp)
    adv.Advect(dt)
    out = adv.fieldSL.vals
    assert rel(out, s["second_out"]) < REF_TOL
    om = oracle.Mesh(int(nx), int(ny), int(N), (0.0, 0.0), (2.0, 1.0), (True, False),
                     accurate=True)
    acc = om.advect(s["second_field"], s["second_vel"], dt, field_prev=s["second_field_prev"],
                    vel_prev=s["second_vel_prev"])
    assert rel(out, acc) < ACC_TOL


@pytest.mark.parametrize("N", [3, 4, 5, 6, 7, 8])
def test_first_order_vs_oracle_all_orders(segpu, oracle, N):
    rng = np.random.default_rng(N)
    nx, ny = 6, 5
    om = oracle.Mesh(nx, ny, N)
    X = om.verts()
    vel = taylor_green(X) + 0.05 * rng.standard_normal((om.nv, 2))
    vel = om.periodic_update(vel, ndofs=2)
    phi = np.sin(2 * np.pi * X[:, 0]) * np.cos(2 * np.pi * X[:, 1]) + 0.01 * rng.standard_normal(om.nv)
    phi = om.periodic_update(phi)
    dt = 2.0 * min(1.0 / nx, 1.0 / ny) / np.sqrt((vel ** 2).sum(1).max())
    ref = om.advect(phi, vel, dt)
    dep, depel = om.departure_first(vel, dt)
    oa = oracle.Mesh(nx, ny, N, accurate=True)
    acc = oa.advect(phi, vel, dt)
    _, depel_acc = oa.departure_first(vel, dt)
    m = make(segpu, nx, ny, N)
    f, v = segpu.Field("phi", m, 1, None), segpu.Field("vel", m, 2, None)
    f.vals, v.vals = phi, vel
    adv = segpu.Advector(f, v)
    adv.record_departures()
    adv.Advect(dt)
    out = adv.fieldSL.vals
    assert rel(out, ref) < REF_TOL
    assert rel(out, acc) < ACC_TOL
    el, xy = adv.departures()
    assert np.array_equal(el, depel_acc)
    mism = np.nonzero(el != depel)[0]
    assert len(mism) == 0, (len(mism), xy[mism[:5]], dep[mism[:5]])
    # the element search itself is bit-exact on the GPU's own departure points
    oel, _ = om.global_to_local(xy)
    assert np.array_equal(oel, el)


def test_second_order_vs_oracle_channel(segpu, oracle):
    rng = np.random.default_rng(7)
    nx, ny, N = 12, 6, 6
    lo, hi = (0.0, 0.0), (2.0, 1.0)
    om = oracle.Mesh(nx, ny, N, lo, hi, (True, False))
    X = om.verts()
    u = np.stack([0.5 + np.sin(np.pi * X[:, 1]) ** 2, 0.3 * np.sin(np.pi * X[:, 0]) * np.sin(np.pi * X[:, 1])], 1)
    up = u * (1 + 0.02 * rng.standard_normal((om.nv, 1)))
    up[:, 1] *= np.sin(np.pi * X[:, 1]) ** 2
    u, up = om.periodic_update(u, 2), om.periodic_update(up, 2)
    psi = om.periodic_update(np.cos(np.pi * X[:, 0]) * np.sin(2 * np.pi * X[:, 1]))
    psip = om.periodic_update(psi + 0.01 * rng.standard_normal(om.nv))
    dt = 1.5 * (2.0 / nx) / np.abs(u).max()
    ref = om.advect(psi, u, dt, field_prev=psip, vel_prev=up)
    x1, e1, x2, e2 = om.departure_second(u, up, dt)
    oa = oracle.Mesh(nx, ny, N, lo, hi, (True, False), accurate=True)
    acc = oa.advect(psi, u, dt, field_prev=psip, vel_prev=up)
    m = make(segpu, nx, ny, N, lo, hi, (True, False))
    f, fp = segpu.Field("psi", m, 1, None), segpu.Field("psiPrev", m, 1, None)
    v, vp = segpu.Field("vel", m, 2, None), segpu.Field("velPrev", m, 2, None)
    f.vals, fp.vals, v.vals, vp.vals = psi, psip, u, up
    adv = segpu.Advector(f, v, fp, vp)
    adv.record_departures()
    adv.Advect(dt)
    out = adv.fieldSL.vals
    assert rel(out, ref) < REF_TOL
    assert rel(out, acc) < ACC_TOL
    el, xy = adv.departures()
    nv = om.nv
    assert np.array_equal(el[:nv], e1) and np.array_equal(el[nv:], e2)


def test_config1_size_departures_bit_exact(segpu, oracle):
    """64x64, p=8, Taylor-Green at Courant 2 (the SL benchmark mesh): every
    departure element equals the reference's; values within tolerance."""
    nx = ny = 64
    N = 8
    om = oracle.Mesh(nx, ny, N)
    X = om.verts()
    vel = taylor_green(X)
    rng = np.random.default_rng(11)
    phi = np.zeros(om.nv)
    for c in rng.uniform(0, 1, size=(4, 2)):
        phi += np.exp(-((X[:, 0] - c[0]) ** 2 + (X[:, 1] - c[1]) ** 2) / 0.05 ** 2)
    dt = om.calc_time_step(vel, 2.0)
    ref = om.advect(phi, vel, dt, nthreads=8)
    _, depel = om.departure_first(vel, dt)
    acc = oracle.Mesh(nx, ny, N, accurate=True).advect(phi, vel, dt, nthreads=8)
    m = make(segpu, nx, ny, N)
    f, v = segpu.Field("phi", m, 1, None), segpu.Field("vel", m, 2, None)
    f.vals, v.vals = phi, vel
    assert abs(segpu.CalcTimeStep(v, 2.0) - dt) <= 1e-15 * dt
    adv = segpu.Advector(f, v)
    adv.record_departures()
    adv.Advect(dt)
    out = adv.fieldSL.vals
    assert rel(out, ref) < REF_TOL
    assert rel(out, acc) < ACC_TOL
    el, _ = adv.departures()
    assert np.array_equal(el, depel)


def test_advect_rejects_low_order_and_mismatch(segpu):
    m2 = make(segpu, 4, 4, 2)
    f, v = segpu.Field("f", m2, 1, None), segpu.Field("v", m2, 2, None)
    with pytest.raises(segpu.SEError) as e:
        segpu.Advector(f, v)
    assert e.value.code == segpu.SE_ERR_UNSUPPORTED
    m = make(segpu, 4, 4, 4)
    f4, s4 = segpu.Field("f", m, 1, None), segpu.Field("s", m, 1, None)
    with pytest.raises(segpu.SEError):
        segpu.Advector(f4, s4)  # velocity must have 2 components


def test_integrate_matches_oracle(segpu, oracle, golden):
    g = golden["mesh"]
    for tag in ("pp", "px", "nn"):
        p = g[f"{tag}_params"]
        m = segpu.Mesh("m", [int(p[0]), int(p[1])], "legendre", int(p[2]), [p[3], p[4]],
                       [p[5], p[6]], [bool(p[7]), bool(p[8])])
        f = segpu.Field("f", m, 1, None)
        f.vals = g[f"{tag}_field"]
        ref = g[f"{tag}_integrate"][0]
        assert abs(f.Integrate(0) - ref) <= 1e-12 * np.abs(g[f"{tag}_field"]).sum()


@pytest.mark.parametrize("tag", ["pp", "px", "nn", "channel"])
def test_gen_vel_bit_exact(segpu, oracle, golden, tag):
    """GenVel (TwoLayerQGEqn::GenVel): (-d psi/dy, d psi/dx) at every vertex,
    bit-exact against the oracle's InterpDerivsGlobal (itself pinned to the
    reference's compiled code), on the fixture meshes and on the full-size
    config-2 channel (128 x 64 elements, p=6, periodic in x, walls in y)."""
    if tag == "channel":
        nx, ny, N, lo, hi, per = 128, 64, 6, (0.0, 0.0), (2.0, 1.0), (True, False)
    else:
        p = golden["mesh"][f"{tag}_params"]
        nx, ny, N = int(p[0]), int(p[1]), int(p[2])
        lo, hi, per = (p[3], p[4]), (p[5], p[6]), (bool(p[7]), bool(p[8]))
    om = oracle.Mesh(nx, ny, N, lo, hi, per)
    X = om.verts()
    psi = np.sin(2.1 * X[:, 0] + 0.3) * np.cos(3.3 * X[:, 1]) + 0.05 * X[:, 0] * X[:, 1]
    psi = om.periodic_update(psi)
    ref = om.interp_derivs_global(psi, X)
    m = make(segpu, nx, ny, N, lo, hi, per)
    f = segpu.Field("psi", m, 1, None)
    f.vals = psi
    vel = segpu.GenVel(f).vals.reshape(-1, 2)
    assert np.array_equal(vel[:, 0], -ref[:, 1])
    assert np.array_equal(vel[:, 1], ref[:, 0])


def test_gen_vel_rejects_bad_fields(segpu):
    m = make(segpu, 4, 4, 4)
    with pytest.raises(segpu.SEError):
        segpu.GenVel(segpu.Field("v", m, 2, None))  # psi must be scalar
    psi = segpu.Field("psi", m, 1, None)
    v2 = segpu.Field("v", make(segpu, 5, 4, 4), 2, None)
    with pytest.raises(segpu.SEError):
        segpu._check(segpu.load_library().se_field_gen_vel(psi._h, v2._h))
