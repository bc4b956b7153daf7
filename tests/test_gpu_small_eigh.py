"""Device eigensolver of the Davidson Rayleigh-Ritz step (lowest k eigenpairs of a small Hermitian
matrix: Householder tridiagonalisation, Sturm multisection, inverse iteration) against numpy's
eigvalsh on spectra that stress it: random (even and odd sizes), exactly and nearly degenerate, already
diagonal, bordered diagonal (the shape of a grown projected matrix), zero, and the largest supported
size."""
import numpy as np
import pytest

from xatu_b200 import _lib as L

pytestmark = pytest.mark.gpu


def _solve(A, k):
    m = A.shape[0]
    T = np.asfortranarray(A.astype(np.complex128))
    theta = np.zeros(k)
    Y = np.zeros((m, k), dtype=np.complex128, order="F")
    st = L.lib().xatu_selftest_small_eigh(0, m, k, L.ptr(T), L.ptr(theta), L.ptr(Y), None)
    assert st == L.XATU_OK, st
    return theta, Y


def _unitary(rng, m):
    q, _ = np.linalg.qr(rng.standard_normal((m, m)) + 1j * rng.standard_normal((m, m)))
    return q


def _cases():
    rng = np.random.default_rng(2024)
    out = []
    for m in (1, 2, 3, 12, 24, 41, 48, 63, 64, 65, 112):
        B = rng.standard_normal((m, m)) + 1j * rng.standard_normal((m, m))
        out.append((f"random{m}", (B + B.conj().T) / 2, min(m, 12)))
    m = 48
    Q = _unitary(rng, m)
    ev = np.sort(np.concatenate([np.repeat(np.linspace(-0.006, 0.02, 8), 2), rng.uniform(0.5, 6, m - 16)]))
    out.append(("twofold", (Q * ev) @ Q.conj().T, 12))
    ev = np.sort(np.concatenate([np.repeat([0.1], 6), rng.uniform(0.5, 6, m - 6)]))
    out.append(("sixfold", (Q * ev) @ Q.conj().T, 12))
    ev = np.sort(np.concatenate([1e-12 * np.arange(12), rng.uniform(0.5, 6, m - 12)]))
    out.append(("near_degenerate", (Q * ev) @ Q.conj().T, 12))
    out.append(("diagonal", np.diag(np.repeat(np.arange(24.0), 2)).astype(complex), 12))
    A = np.diag(np.sort(rng.uniform(-0.01, 3, m))).astype(complex)
    Bb = (rng.standard_normal((36, 12)) + 1j * rng.standard_normal((36, 12))) * 1e-3
    A[:36, 36:] = Bb
    A[36:, :36] = Bb.conj().T
    out.append(("bordered", A, 12))
    out.append(("zero", np.zeros((8, 8), complex), 4))
    m = 112
    B = rng.standard_normal((m, m)) + 1j * rng.standard_normal((m, m))
    out.append(("k56_m112", (B + B.conj().T) / 2, 56))
    return out


@pytest.mark.parametrize("name,A,k", _cases(), ids=[c[0] for c in _cases()])
def test_small_eigh_lowest(name, A, k):
    theta, Y = _solve(A, k)
    w = np.linalg.eigvalsh(A)[:k]
    scale = max(1.0, np.abs(w).max())
    assert np.all(np.diff(theta) >= -1e-14 * scale)
    assert np.abs(theta - w).max() <= 1e-12 * scale, (theta, w)
    assert np.abs(A @ Y - Y * theta).max() <= 1e-11 * scale
    assert np.abs(Y.conj().T @ Y - np.eye(k)).max() <= 1e-11


def test_small_eigh_rejects_oversize():
    m = 113
    T = np.zeros((m, m), dtype=np.complex128, order="F")
    theta = np.zeros(4)
    Y = np.zeros((m, 4), dtype=np.complex128, order="F")
    assert L.lib().xatu_selftest_small_eigh(0, m, 4, L.ptr(T), L.ptr(theta), L.ptr(Y), None) == L.XATU_ERR_INVALID
