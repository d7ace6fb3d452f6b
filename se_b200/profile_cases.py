"""Single-kernel cases for profiling the library with ncu.

    python -m se_b200.profile_cases apply   # operator apply, 64x64 elements, p=8
    python -m se_b200.profile_cases sl      # first-order SL advection, same mesh
    python -m se_b200.profile_cases cg      # persistent Jacobi-PCG solve, same mesh
    python -m se_b200.profile_cases fdm     # one FDM solve (a CUDA graph)

Each case builds the bench's 64x64-element, p=8, doubly periodic mesh and
fields and launches the kernel a few times directly (not inside a graph), so
that ncu can capture individual launches. Prints one line with the mean
device time of the launches (CUDA events).
"""
from __future__ import annotations

import sys

import numpy as np


def main(case: str, reps: int = 3) -> None:
    import torch

    from . import segpu as S

    S.load_library()
    torch.cuda.init()
    nx, p = 64, 8
    m = S.Mesh("m", [nx, nx], "legendre", p, [0.0, 0.0], [1.0, 1.0], [True, True])
    X = m.verts
    x, y = X[:, 0], X[:, 1]
    vel = np.stack([-np.sin(np.pi * x) ** 2 * np.sin(2 * np.pi * y),
                    np.sin(np.pi * y) ** 2 * np.sin(2 * np.pi * x)], 1)
    phi0 = np.exp(-((x - 0.4) ** 2 + (y - 0.6) ** 2) / 0.05 ** 2)
    bc = S.BCs(False, False, False, False, m)
    phi, v, u = S.Field("phi", m, 1, bc), S.Field("v", m, 2, None), S.Field("u", m, 1, bc)
    phi.vals, v.vals = phi0, vel
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(reps)]
    if case == "sl":
        adv = S.Advector(phi, v)
        dt = S.CalcTimeStep(v, 2.0)
        for a, b in ev:
            a.record()
            adv.Advect(dt)
            b.record()
    elif case in ("apply", "cg", "fdm"):
        method = S.METHOD_FDM if case == "fdm" else S.METHOD_CG
        h = S.HelmholtzEqn(u, phi, -1.0, -1.0, 1.0, 0,
                           S.solver_opts(rtol=1e-10, mode=S.MODE_EXACT, method=method))
        n = h.vecSize
        xin = torch.randn(n, dtype=torch.float64, device="cuda")
        yout = torch.empty_like(xin)
        for a, b in ev:
            a.record()
            if case == "apply":
                h.apply(xin.data_ptr(), yout.data_ptr())
            else:
                h.Solve("helm_")
            b.record()
    else:
        raise SystemExit(f"unknown case {case!r}")
    torch.cuda.synchronize()
    ms = [a.elapsed_time(b) for a, b in ev]
    print(f"{case}: mean {np.mean(ms):.4f} ms over {reps} launches", flush=True)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "apply")
