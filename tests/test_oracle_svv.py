"""The spectral vanishing viscosity operator (SVV, src/base/SVV.cpp) in the
oracle, pinned against the reference, and the Kronecker form the GPU path
applies.

The oracle restates SVV::AssembleElement literally: dense (N+1)^2-sized
modal transform B, weights W, the inverses (B^T W B)^-1 and M^-1, the
filter Q, the derivative matrices and the products, with Lyy formed from
the x-derivative as the reference forms it. Its inverse is Gauss-Jordan
with partial pivoting where the reference's is full pivoting, so the
element matrices agree to rounding (1e-12 relative), not bit for bit.

The GPU path uses the factored form of the same matrix: with the filter
F = B1 diag(q) B1^-1 on one axis (B1 the 1-D modal basis at the GLL nodes,
q(k) = exp(-(N-k)^2/(mN-k)^2 / 2) for k > mN, else 0), S = (F D)^T W1 (F D)
and T = F^T W1 F, the element matrix is 2 c detJ (T_y kron S_x)."""
import numpy as np
import pytest

CASES = [(4, 2), (6, 3), (8, 4), (7, 3), (3, 1), (10, 5)]


def modal_coeffs(N):
    """Monomial coefficients of Legendre::ModalBasis (src/base/Legendre.cpp:307-335)."""
    Pn = [np.zeros(N + 2) for _ in range(N + 1)]
    Pn[0][0] = 1.0
    if N >= 1:
        Pn[1][1] = 2.0
    a = 1.0
    for n in range(2, N + 1):
        c1 = 2 * n * (2 * a + n) * (2 * a + 2 * n - 2)
        c2 = (2 * a + 2 * n - 1) * (2 * a + 2 * n) * (2 * a + 2 * n - 2) / c1
        c3 = 2 * (a + n - 1) * (a + n - 1) * (2 * a + 2 * n) / c1
        Pn[n][1:] += c2 * Pn[n - 1][:-1]
        Pn[n] -= c3 * Pn[n - 2]
    modal = np.zeros((N + 1, N + 2))
    modal[0, :2] = [0.5, 0.5]
    modal[1, :2] = [0.5, -0.5]
    for i in range(2, N + 1):
        modal[i, :N] += 0.25 * Pn[i - 2][:N]
        modal[i, 2:] -= 0.25 * Pn[i - 2][:N]
    return modal


def kron_form(oracle, N, mN, c, hx, hy):
    x, w, dC, _ = oracle.gll(N)
    modal = modal_coeffs(N)
    B = np.array([[np.polyval(modal[k][::-1], xa) for k in range(N + 1)] for xa in x])
    q = np.array([np.exp(-((N - k) ** 2) / ((mN - k) ** 2) / 2) if k > mN else 0.0
                  for k in range(N + 1)])
    F = B @ np.diag(q) @ np.linalg.inv(B)
    FD = F @ dC.reshape(N + 1, N + 1)
    S = FD.T @ np.diag(w) @ FD
    T = F.T @ np.diag(w) @ F
    return 2 * c * (hx / 2) * (hy / 2) * np.kron(T, S)


def fixture_mesh(oracle, golden, N, use_ref=False):
    p = golden["svv"]["params"]
    return oracle.Mesh(int(p[0]), int(p[1]), N, (p[2], p[3]), (p[4], p[5]), (False, False),
                       use_ref=use_ref)


@pytest.mark.parametrize("N", [4, 6, 8])
def test_svv_oracle_matches_reference_fixture(oracle, golden, N):
    ref = golden["svv"][f"elmat_{N}"]
    got = fixture_mesh(oracle, golden, N).svv_element(4, 0.7, N // 2)
    assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()


@pytest.mark.parametrize("N,mN", CASES)
def test_svv_oracle_matches_reference_live(oracle, N, mN):
    if not oracle.ref_available():
        pytest.skip("reference library not built here")
    args = (4, 3, N, (-0.3, 0.1), (1.1, 0.9), (True, False))
    om, rm = oracle.Mesh(*args), oracle.Mesh(*args, use_ref=True)
    for el in (0, 7, 11):
        a, b = om.svv_element(el, 0.35, mN), rm.svv_element(el, 0.35, mN)
        assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max()


@pytest.mark.parametrize("N,mN", CASES)
def test_svv_kronecker_form(oracle, N, mN):
    lo, hi, ne = (0.0, -0.5), (1.5, 0.3), (3, 2)
    m = oracle.Mesh(ne[0], ne[1], N, lo, hi, (False, False))
    E = m.svv_element(4, 0.7, mN)
    K = kron_form(oracle, N, mN, 0.7, (hi[0] - lo[0]) / ne[0], (hi[1] - lo[1]) / ne[1])
    assert np.abs(E - K).max() <= 1e-11 * np.abs(E).max()
    # symmetric, positive semi-definite, constants in its null space
    assert np.abs(E - E.T).max() <= 1e-14 * np.abs(E).max() * E.shape[0]
    assert np.abs(E.sum(1)).max() <= 1e-13 * np.abs(E).max() * E.shape[0]
    assert np.linalg.eigvalsh(0.5 * (E + E.T)).min() >= -1e-12 * np.abs(E).max()


def test_svv_cutoff_at_order_is_zero(oracle):
    m = oracle.Mesh(2, 2, 5, (0.0, 0.0), (1.0, 1.0), (False, False))
    assert not np.any(m.svv_element(0, 1.0, 5))
