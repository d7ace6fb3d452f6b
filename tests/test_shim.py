"""The C++ shim (include/segpu.hpp) that gives reference callers the
reference's class names over the C-ABI: compiled by g++ against segpu.h and
linked with libsegpu.so, so that the shim cannot drift from the header.

The CPU test builds it and runs the options parser, a Mesh and a Field
construction, which must fail with the library's message when no CUDA
device is present;
the GPU test runs an advection and a Helmholtz solve through the shim on
fields the test writes, and compares the result with the same calls through
the Python binding (identical: the same kernels on the same inputs)."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def shim_exe(segpu, tmp_path_factory):
    out = str(tmp_path_factory.mktemp("shim") / "shim_main")
    lib = os.path.join(ROOT, "se_b200")
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "shim", "shim_main.cpp"), "-o", out, "-L", lib, "-lsegpu",
           f"-Wl,-rpath,{lib}"]
    subprocess.run(cmd, check=True)
    return out


def test_shim_compiles_and_links_and_parses_options(shim_exe):
    r = subprocess.run([shim_exe, "cpu"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.splitlines()
    assert lines[0].startswith("version segpu")
    assert lines[1] == f"opts rtol 1e-09 max_it 77 method 1"
    assert lines[2] == "mesh 625 vertices"
    import torch
    if not torch.cuda.is_available():
        assert lines[3].startswith("field refused: ") and len(lines[3]) > len("field refused: ")


@pytest.mark.gpu
def test_shim_solve_matches_python_binding(shim_exe, segpu, tmp_path):
    S = segpu
    m = S.Mesh("m", [8, 8], "legendre", 6, [0.0, 0.0], [1.0, 1.0], [True, True])
    X = m.verts
    x, y = X[:, 0], X[:, 1]
    phi0 = np.exp(-((x - 0.3) ** 2 + (y - 0.6) ** 2) / 0.0025)
    vel = np.stack([-np.sin(np.pi * x) ** 2 * np.sin(2 * np.pi * y),
                    np.sin(np.pi * y) ** 2 * np.sin(2 * np.pi * x)], 1)
    fields = tmp_path / "fields.bin"
    np.concatenate([phi0, vel.ravel()]).astype("<f8").tofile(fields)
    r = subprocess.run([shim_exe, "gpu", str(fields)], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.splitlines()
    its = int(lines[0].split()[1])
    got = np.array([float(v) for v in lines[1:]])
    bc = S.BCs(False, False, False, False, m)
    phi, v, u = S.Field("phi", m, 1, bc), S.Field("vel", m, 2, None), S.Field("u", m, 1, bc)
    phi.vals, v.vals = phi0, vel
    adv = S.Advector(phi, v)
    adv.Advect(0.01)
    phi.Copy(adv.fieldSL)
    h = S.HelmholtzEqn(u, phi, -1.0, -1.0, 1.0, 0, S.solver_opts(rtol=1e-10))
    st = h.Solve("helm_")
    # the same inputs through the same library: the same result
    assert its == st["its"]
    assert np.array_equal(got, u.vals)
