"""Host-side checks of the product library that need no GPU: it loads, it
exports every entry point include/segpu.h declares, and its host tables (GLL
nodes/weights/derivatives, vertex coordinates, boundary-condition maps,
options parsing) equal the reference's bit for bit."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "segpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(se_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol(segpu):
    lib = ctypes.CDLL(segpu.LIB_PATH)
    names = declared_symbols()
    assert len(names) > 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) == set(segpu.SIGNATURES), set(names) ^ set(segpu.SIGNATURES)


def _mesh(S, p):
    nx, ny, N = int(p[0]), int(p[1]), int(p[2])
    return S.Mesh("m", [nx, ny], "legendre", N, [p[3], p[4]], [p[5], p[6]],
                  [bool(p[7]), bool(p[8])])


@pytest.mark.parametrize("N", range(2, 13))
def test_gll_tables_bit_exact(segpu, golden, N):
    m = segpu.Mesh("m", [2, 2], "legendre", N, [0, 0], [1, 1], [True, True])
    a, w, dc = m.gll()
    g = golden["gll"]
    assert np.array_equal(a, g[f"abcissa_{N}"])
    assert np.array_equal(w, g[f"weights_{N}"])
    assert np.array_equal(dc, g[f"dC_{N}"])


@pytest.mark.parametrize("tag", ["pp", "px", "nn"])
def test_vertices_and_bc_maps_bit_exact(segpu, golden, tag):
    g = golden["mesh"]
    m = _mesh(segpu, g[f"{tag}_params"])
    assert np.array_equal(m.verts, g[f"{tag}_verts"])
    for k in range(int(g[f"{tag}_nbc"][0])):
        bc = [bool(b) for b in g[f"{tag}_bc{k}"]]
        b = segpu.BCs(*bc, m)
        f2v, v2f = b.maps()
        assert np.array_equal(f2v, g[f"{tag}_f2v{k}"]), bc
        assert np.array_equal(v2f, g[f"{tag}_v2f{k}"]), bc


def test_bc_configuration_errors(segpu):
    m = segpu.Mesh("m", [3, 3], "legendre", 4, [0, 0], [1, 1], [True, True])
    with pytest.raises(segpu.SEError) as e:
        segpu.BCs(True, True, False, False, m)
    assert e.value.code == segpu.SE_ERR_ARG
    my = segpu.Mesh("m", [3, 3], "legendre", 4, [0, 0], [1, 1], [False, True])
    with pytest.raises(segpu.SEError) as e:
        segpu.BCs(False, False, False, False, my)
    assert e.value.code == segpu.SE_ERR_UNSUPPORTED
    with pytest.raises(segpu.SEError):
        segpu.Mesh("m", [3, 3], "chebyshev", 4, [0, 0], [1, 1], [True, True])
    with pytest.raises(segpu.SEError) as e:
        segpu.Mesh("m", [3, 3], "legendre", 13, [0, 0], [1, 1], [True, True])
    assert e.value.code == segpu.SE_ERR_UNSUPPORTED
    with pytest.raises(segpu.SEError):
        segpu.Mesh("m", [0, 3], "legendre", 4, [0, 0], [1, 1], [True, True])


def test_solver_options_parse(segpu):
    o = segpu.solver_opts("helm_", "-helm_ksp_type cg -helm_pc_type jacobi -helm_ksp_rtol 1e-12 "
                          "-helm_ksp_max_it 77 -poisson_ksp_rtol 3 -helm_ksp_norm_type natural")
    assert o.rtol == 1e-12 and o.max_it == 77 and o.norm_type == segpu.NORM_NATURAL
    d = segpu.solver_opts()
    assert d.rtol == 1e-5 and d.max_it == 10000 and d.atol == 1e-50 and d.dtol == 1e5
    with pytest.raises(segpu.SEError) as e:
        segpu.solver_opts("helm_", "-helm_ksp_type gmres")
    assert e.value.code == segpu.SE_ERR_UNSUPPORTED
    o = segpu.solver_opts("helm_", "-helm_pc_type fdm -helm_precision fp64_tc")
    assert o.method == segpu.METHOD_FDM and o.precision == segpu.PREC_FP64_TC
    o = segpu.solver_opts("helm_", "-helm_pc_type fdm -helm_precision mixed")
    assert o.precision == segpu.PREC_MIXED
    o = segpu.solver_opts("helm_", "-helm_ksp_type cg -helm_precision fp16")
    assert o.method == segpu.METHOD_CG and o.precision == segpu.PREC_FP16
    with pytest.raises(segpu.SEError) as e:
        segpu.solver_opts("helm_", "-helm_precision fp8")
    assert e.value.code == segpu.SE_ERR_UNSUPPORTED


def test_no_device_fails_loudly(segpu):
    """Without a CUDA device, field creation must fail (no CPU fallback)."""
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a CUDA device is present")
    except Exception:
        pass
    m = segpu.Mesh("m", [2, 2], "legendre", 4, [0, 0], [1, 1], [True, True])
    with pytest.raises(segpu.SEError) as e:
        segpu.Field("f", m, 1, None)
    assert e.value.code == segpu.SE_ERR_CUDA
