"""The continuous-batching server (se_server_*): each request's result is the
same alone and in a concurrent mix, and the same as the direct API path
(tolerance: bit-identical -- the kernels are deterministic); admission works
with fewer slots than requests and with a budget smaller than one request."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def requests(S):
    rng = np.random.default_rng(9)
    reqs = []
    for nx, ny, p, per, bcs in [(8, 8, 4, (1, 1), (0, 0, 0, 0)), (12, 10, 6, (1, 1), (0, 0, 0, 0)),
                                (16, 16, 8, (1, 1), (0, 0, 0, 0)), (10, 6, 5, (1, 0), (1, 1, 0, 0)),
                                (7, 9, 6, (0, 0), (1, 1, 1, 1))]:
        m = S.Mesh("m", [nx, ny], "legendre", p, [0, 0], [1, 1], list(per))
        X = m.verts
        f = np.sin(2 * np.pi * X[:, 0] + rng.uniform()) * np.cos(2 * np.pi * X[:, 1])
        aux = 0.2 * np.cos(X[:, 0]) if not per[1] else None
        reqs.append(dict(kind=S.REQ_HELMHOLTZ, nEls=(nx, ny), N=p, lo=(0, 0), hi=(1, 1),
                         periodic=per, field_in=f, aux=aux, bcs=bcs, c=-2.0, nu=-1.0, dt=1.0))
    for nx, p, steps in [(8, 6, 10), (10, 5, 4), (12, 8, 10)]:
        m = S.Mesh("m", [nx, nx], "legendre", p, [0, 0], [1, 1], [True, True])
        X = m.verts
        vel = np.stack([-np.sin(np.pi * X[:, 0]) ** 2 * np.sin(2 * np.pi * X[:, 1]),
                        np.sin(np.pi * X[:, 1]) ** 2 * np.sin(2 * np.pi * X[:, 0])], 1)
        phi = np.exp(-((X[:, 0] - 0.4) ** 2 + (X[:, 1] - 0.6) ** 2) / 0.01)
        reqs.append(dict(kind=S.REQ_ADVECT, nEls=(nx, nx), N=p, lo=(0, 0), hi=(1, 1),
                         periodic=(1, 1), field_in=phi, aux=vel, steps=steps, sl_dt=0.02))
    return reqs


def test_results_same_alone_in_mix_and_direct(segpu):
    reqs = requests(segpu)
    srv = segpu.Server(slots=4, device_gib=8.0)
    alone = []
    for r in reqs:
        out, res = srv.wait(srv.submit(**r))
        assert res["status"] == 0
        if r["kind"] == segpu.REQ_HELMHOLTZ:
            assert res["reason"] == 2
        alone.append(out)
    order = list(range(len(reqs))) * 3
    np.random.default_rng(1).shuffle(order)
    tickets = [(k, srv.submit(**reqs[k])) for k in order]
    for k, t in tickets:
        out, res = srv.wait(t)
        assert res["status"] == 0 and res["latency_ms"] >= res["queued_ms"] >= 0
        assert np.array_equal(out, alone[k])
    srv.close()
    # the direct API path computes the same numbers
    for r, got in zip(reqs, alone):
        m = segpu.Mesh("m", list(r["nEls"]), "legendre", r["N"], list(r["lo"]), list(r["hi"]),
                       [bool(x) for x in r["periodic"]])
        if r["kind"] == segpu.REQ_HELMHOLTZ:
            b = segpu.BCs(*[bool(x) for x in r["bcs"]], m)
            u, f = segpu.Field("u", m, 1, b), segpu.Field("f", m, 1, b)
            f.vals = r["field_in"]
            u.vals = r["aux"] if r["aux"] is not None else 0.0
            h = segpu.HelmholtzEqn(u, f, r["c"], r["nu"], r["dt"], 0,
                                   segpu.solver_opts(rtol=1e-10, mode=segpu.MODE_EXACT,
                                                     method=segpu.METHOD_FDM))
            h.Solve("helm_")
            assert np.array_equal(u.vals, got)
        else:
            phi, v = segpu.Field("phi", m, 1, None), segpu.Field("v", m, 2, None)
            phi.vals, v.vals = r["field_in"], r["aux"]
            adv = segpu.Advector(phi, v)
            for _ in range(r["steps"]):
                adv.Advect(r["sl_dt"])
                phi.Copy(adv.fieldSL)
            assert np.array_equal(phi.vals, got)


def test_admission_with_few_slots_and_a_tiny_budget(segpu):
    reqs = requests(segpu)
    srv = segpu.Server(slots=2, device_gib=1e-4)  # smaller than any request
    tickets = [srv.submit(**r) for r in reqs * 2]
    outs = [srv.wait(t) for t in tickets]
    assert all(res["status"] == 0 for _, res in outs)
    for (a, _), (b, _) in zip(outs[: len(reqs)], outs[len(reqs):]):
        assert np.array_equal(a, b)
    srv.close()


@pytest.mark.parametrize("prec", ["PREC_MIXED", "PREC_FP64_TC"])
def test_mixed_precision_results_same_alone_and_in_mix(segpu, prec):
    """The tensor-core solve precisions through the lean request path
    (request / submit_request / wait_request, the serving benchmark's
    client): each Helmholtz result is bit-identical alone and in a shuffled
    concurrent mix, and within 1e-9 of the FP64 solve."""
    S = segpu
    opts = S.solver_opts(rtol=1e-10, mode=S.MODE_EXACT, method=S.METHOD_FDM,
                         precision=getattr(S, prec))
    srv = S.Server(slots=4, device_gib=8.0)
    reqs = [r for r in requests(S) if r["kind"] == S.REQ_HELMHOLTZ]
    built = []
    for r in reqs:
        f = np.ascontiguousarray(r["field_in"], dtype=np.float64)
        aux = None if r["aux"] is None else np.ascontiguousarray(r["aux"], dtype=np.float64)
        outs = [np.zeros(len(f)) for _ in range(4)]
        reqs_k = [srv.request(r["kind"], r["nEls"], r["N"], r["lo"], r["hi"], r["periodic"], f,
                              aux, bcs=r["bcs"], c=r["c"], nu=r["nu"], dt=r["dt"], opts=opts,
                              out=o) for o in outs]
        built.append((f, aux, outs, reqs_k))
    alone = []
    for f, aux, outs, rk in built:
        res = srv.wait_request(srv.submit_request(rk[0]))
        assert res.status == 0 and res.reason == 2
        alone.append(outs[0].copy())
    order = [(k, c) for k in range(len(built)) for c in range(1, 4)]
    np.random.default_rng(3).shuffle(order)
    tickets = [(k, c, srv.submit_request(built[k][3][c])) for k, c in order]
    for k, c, t in tickets:
        res = srv.wait_request(t)
        assert res.status == 0 and res.reason == 2
        assert np.array_equal(built[k][2][c], alone[k])
    srv.close()
    # against the FP64 solve of the same systems
    fp = S.Server(slots=2, device_gib=8.0)
    for r, got in zip(reqs, alone):
        out, res = fp.wait(fp.submit(**r))
        assert res["status"] == 0
        assert np.abs(out - got).max() <= 1e-9 * np.abs(out).max()
    fp.close()
