"""Generate the golden fixtures in tests/golden/ from the reference itself.

Runs the reference's own src/base code, compiled unmodified into
oracle/_ref/libseref.so by ``make -C oracle ref`` (needs the SE checkout,
read-only, named by the SE_REFERENCE_SRC environment variable). The fixtures
pin the oracle restatement and the product's host tables on machines
without the checkout.

    SE_REFERENCE_SRC=<SE checkout> python tests/golden/make_golden.py

The reference publishes no golden vectors or known-answer tests of its own;
these are seeded synthetic cases with the shapes the reference runs.
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def taylor_green(X, amp=1.0):
    x, y = X[:, 0], X[:, 1]
    return np.stack([-amp * np.sin(np.pi * x) ** 2 * np.sin(2 * np.pi * y),
                     amp * np.sin(np.pi * y) ** 2 * np.sin(2 * np.pi * x)], 1)


def blobs(X, centres, width):
    f = np.zeros(len(X))
    for c in centres:
        f += np.exp(-((X[:, 0] - c[0]) ** 2 + (X[:, 1] - c[1]) ** 2) / width ** 2)
    return f


def edge_points(m: O.Mesh, rng, n):
    """Points on and within a few ulps / 1e-12 of element edges and GLL nodes."""
    a, _, _, _ = O.gll(m.N, use_ref=True)
    dx = [(m.hi[k] - m.lo[k]) / (m.nx if k == 0 else m.ny) for k in range(2)]
    pts = []
    for _ in range(n):
        p = []
        for k in range(2):
            ne = m.nx if k == 0 else m.ny
            e = rng.integers(0, ne + 1)
            base = m.lo[k] + e * dx[k]
            kind = rng.integers(0, 4)
            if kind == 0:
                off = rng.choice([-1, 1]) * rng.choice([0.0, 1e-12, 1e-12 * (1 + 1e-4), 1e-13, 5e-17])
                v = base + off
            elif kind == 1:
                v = np.nextafter(base, base + rng.choice([-1, 1]) * 1.0)
            elif kind == 2:
                j = rng.integers(0, m.N + 1)
                v = m.lo[k] + min(e, ne - 1) * dx[k] + (a[j] + 1.0) / 2.0 * dx[k]
                v += rng.choice([0.0, 1e-9, -1e-9, 2e-8, 1e-7]) * dx[k] / 2
            else:
                v = rng.uniform(m.lo[k], m.hi[k])
            p.append(min(max(v, m.lo[k]), m.hi[k]))
        pts.append(p)
    return np.array(pts)


def main():
    if not O.ref_available():
        O.build(with_ref=True)
    rng = np.random.default_rng(20241203)

    # GLL tables (src/base/Legendre.cpp:15-95)
    g = {}
    for N in range(2, 13):
        a, w, dc, pj = O.gll(N, use_ref=True)
        g[f"abcissa_{N}"], g[f"weights_{N}"], g[f"dC_{N}"], g[f"Pj_{N}"] = a, w, dc, pj
    np.savez_compressed(os.path.join(OUT, "gll.npz"), **g)

    # Mesh, element search, interpolation, element matrices, FieldRHS, BCs
    d = {}
    cases = [("pp", (6, 5, 5, (-1.0, 0.0), (1.0, 1.5), (True, True))),
             ("px", (7, 4, 4, (0.0, 0.0), (2.0, 1.0), (True, False))),
             ("nn", (3, 4, 6, (-1.0, -1.0), (1.0, 1.0), (False, False)))]
    for tag, (nx, ny, N, lo, hi, per) in cases:
        m = O.Mesh(nx, ny, N, lo, hi, per, use_ref=True)
        d[f"{tag}_params"] = np.array([nx, ny, N, lo[0], lo[1], hi[0], hi[1], per[0], per[1]],
                                      dtype=np.float64)
        d[f"{tag}_verts"] = m.verts()
        v = rng.standard_normal(m.nv)
        vel = rng.standard_normal((m.nv, 2))
        d[f"{tag}_field"], d[f"{tag}_vel"] = v, vel
        pts = np.concatenate([rng.uniform(lo, hi, size=(300, 2)), edge_points(m, rng, 300)])
        d[f"{tag}_pts"] = pts
        el, lc = m.global_to_local(pts)
        d[f"{tag}_el"], d[f"{tag}_lc"] = el, lc
        d[f"{tag}_interp"] = m.interp_global(v, pts)
        d[f"{tag}_interp_vel"] = m.interp_global(vel, pts, ndofs=2)
        d[f"{tag}_derivs"] = m.interp_derivs_global(v, pts)
        d[f"{tag}_integrate"] = np.array([m.integrate(v)])
        els = [0, nx * ny // 2, nx * ny - 1]
        d[f"{tag}_els"] = np.array(els)
        d[f"{tag}_elmat"] = np.stack([m.element_matrix(e, -2.5, -1.0) for e in els])
        d[f"{tag}_elrhs"] = np.stack([m.field_rhs_element(v, e) for e in els])
        bcs_list = ([(False, False, False, False)] if per == (True, True) else
                    [(False, False, False, False), (True, True, False, False),
                     (False, True, False, False)] if per == (True, False) else
                    [(True, True, True, True), (True, False, True, False),
                     (False, False, False, False), (False, True, False, True)])
        for k, bc in enumerate(bcs_list):
            f2v, v2f = m.bcs_maps(*bc)
            d[f"{tag}_bc{k}"] = np.array(bc, dtype=np.int32)
            d[f"{tag}_f2v{k}"], d[f"{tag}_v2f{k}"] = f2v, v2f
        d[f"{tag}_nbc"] = np.array([len(bcs_list)])
    np.savez_compressed(os.path.join(OUT, "mesh.npz"), **d)

    # SL advection: first order on a doubly periodic unit square with a
    # Taylor-Green velocity at Courant number 2; second order on a channel.
    s = {}
    m = O.Mesh(8, 8, 6, (0.0, 0.0), (1.0, 1.0), (True, True), use_ref=True)
    X = m.verts()
    vel = taylor_green(X)
    phi = blobs(X, rng.uniform(0, 1, size=(4, 2)), 0.15)
    dt = 2.0 * (1.0 / 8) / np.sqrt((vel ** 2).sum(1).max())
    s["first_params"] = np.array([8, 8, 6, dt])
    s["first_field"], s["first_vel"] = phi, vel
    s["first_out"] = m.advect(phi, vel, dt)
    dep, el = m.departure_first(vel, dt)
    s["first_dep"], s["first_depel"] = dep, el
    s["first_vel_out"] = m.advect(vel, vel, dt)  # 2-component field (velocity self-advection)

    m2 = O.Mesh(8, 6, 4, (0.0, 0.0), (2.0, 1.0), (True, False), use_ref=True)
    X2 = m2.verts()
    vel2 = np.stack([0.6 + 0.3 * np.sin(np.pi * X2[:, 1]) * np.cos(np.pi * X2[:, 0]),
                     0.2 * np.sin(np.pi * X2[:, 0]) * np.sin(np.pi * X2[:, 1])], 1)
    vel2p = vel2 * 0.97 + 0.01 * rng.standard_normal(vel2.shape) * np.sin(np.pi * X2[:, 1:2])
    psi = np.cos(np.pi * X2[:, 0]) * np.sin(np.pi * X2[:, 1]) + 0.1 * rng.standard_normal(m2.nv)
    psip = psi * 0.99
    dt2 = 0.05
    s["second_params"] = np.array([8, 6, 4, dt2])
    s["second_field"], s["second_field_prev"] = psi, psip
    s["second_vel"], s["second_vel_prev"] = vel2, vel2p
    s["second_out"] = m2.advect(psi, vel2, dt2, field_prev=psip, vel_prev=vel2p)
    np.savez_compressed(os.path.join(OUT, "sl.npz"), **s)

    # SVV element matrices (src/base/SVV.cpp:50-176) at the cutoffs the
    # reference's models use (N/2), one element of a non-square mesh each
    v = {}
    for N in (4, 6, 8):
        m = O.Mesh(3, 2, N, (0.0, -0.5), (1.5, 0.3), (False, False), use_ref=True)
        v[f"elmat_{N}"] = m.svv_element(4, 0.7, N // 2)
    v["params"] = np.array([3, 2, 0.0, -0.5, 1.5, 0.3, 4, 0.7])
    np.savez_compressed(os.path.join(OUT, "svv.npz"), **v)
    for f in ("gll.npz", "mesh.npz", "sl.npz", "svv.npz"):
        print(f, os.path.getsize(os.path.join(OUT, f)))


if __name__ == "__main__":
    main()
