"""Single-kernel cases for profiling the library with ncu.

    python tests/profile_cases.py apply [ne]       # FP64 operator apply
    python tests/profile_cases.py apply_bf16 [ne]  # BF16-in, FP32 operator apply
    python tests/profile_cases.py sl [ne]          # first-order SL advection
    python tests/profile_cases.py sl2 [ne]         # second-order SL advection
    python tests/profile_cases.py cg [ne]          # persistent Jacobi-PCG solve
    python tests/profile_cases.py fdm [ne]         # one FDM solve (a CUDA graph)
    python tests/profile_cases.py fdm_apply [ne]   # the FDM transform: 4 product kernels
    python tests/profile_cases.py fdm_apply_tc [ne]  # the same on the tcgen05 tensor cores (TF32 hi/lo)
    python tests/profile_cases.py residual [ne]    # the refinement residual r = b - A x (double-double)

Each case builds an ne x ne element (default 64, the bench's mesh), order p
(third argument, default 8), doubly periodic mesh and the bench's fields and launches the kernel a few
times directly (not inside a graph), so that ncu can capture individual
launches. Prints one line with the mean device time of the launches (CUDA
events).
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def main(case: str, ne: int = 64, p: int = 8, reps: int = 3) -> None:
    import torch

    from se_b200 import segpu as S

    S.load_library()
    torch.cuda.init()
    nx = ne
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
    if case in ("sl", "sl2"):
        if case == "sl":
            adv = S.Advector(phi, v)
        else:  # second order: previous level = the same fields, shifted / scaled
            phim, vm = S.Field("phim", m, 1, bc), S.Field("vm", m, 2, None)
            phim.vals, vm.vals = np.roll(phi0, 1), 0.98 * vel
            adv = S.Advector(phi, v, phim, vm)
        dt = S.CalcTimeStep(v, 2.0)
        for a, b in ev:
            a.record()
            adv.Advect(dt)
            b.record()
    elif case in ("apply", "apply_bf16", "cg", "fdm", "fdm_apply", "fdm_apply_tc", "residual"):
        method = S.METHOD_FDM if case.startswith("fdm") else S.METHOD_CG
        h = S.HelmholtzEqn(u, phi, -1.0, -1.0, 1.0, 0,
                           S.solver_opts(rtol=1e-10, mode=S.MODE_EXACT, method=method))
        n = h.vecSize
        xin = torch.randn(n, dtype=torch.float64, device="cuda")
        yout = torch.empty_like(xin)
        xb = xin.float().to(torch.bfloat16)
        yf = torch.empty(n, dtype=torch.float32, device="cuda")
        bres = torch.randn(n, dtype=torch.float64, device="cuda")
        for a, b in ev:
            a.record()
            if case == "apply":
                h.apply(xin.data_ptr(), yout.data_ptr())
            elif case == "apply_bf16":
                h.apply_low(xb.data_ptr(), yf.data_ptr(), S.PREC_BF16)
            elif case == "fdm_apply":
                h.fdm_apply(xin.data_ptr(), yout.data_ptr())
            elif case == "fdm_apply_tc":
                h.fdm_apply(xin.data_ptr(), yout.data_ptr(), S.PREC_MIXED)
            elif case == "residual":
                h.residual(xin.data_ptr(), bres.data_ptr(), yout.data_ptr())
            else:
                h.Solve("helm_")
            b.record()
    else:
        raise SystemExit(f"unknown case {case!r}")
    torch.cuda.synchronize()
    ms = [a.elapsed_time(b) for a, b in ev]
    print(f"{case}: mean {np.mean(ms):.4f} ms over {reps} launches", flush=True)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "apply", int(sys.argv[2]) if len(sys.argv) > 2 else 64,
         int(sys.argv[3]) if len(sys.argv) > 3 else 8)
