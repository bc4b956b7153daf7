"""H.X products of the mixed build (the Davidson's inner kernel) against the
oracle's FP64 matrix: CUDA-core kernel and tcgen05 tensor-core kernel.

Tolerance: the split-BF16 planes carry K to ~2^-16 relative and the products
accumulate in FP32, so |dY| <= 2e-5 * max|H| * ||x||_1-ish; the test uses
2e-5 relative to max |Y|."""
import numpy as np
import pytest

from tests.helpers import engine_exciton, model_config, oracle_exciton

pytestmark = pytest.mark.gpu

HX_TOL = 2e-5


def _setup(model, ncell, nbands, params, **kw):
    cfg = model_config(model) if isinstance(model, str) else model
    ex = engine_exciton(cfg, ncell, nbands, params, **kw)
    orc = oracle_exciton(cfg, ncell, nbands, params, **kw)
    ex.upload_bands(orc.eigval, orc.eigvec, orc.eigvalQ, orc.eigvecQ)
    ex.BShamiltonian("mixed")
    return ex, orc.bs_hamiltonian()


def _x(N, nvec, seed=0):
    rng = np.random.default_rng(seed)
    X = rng.normal(size=(N, nvec)) + 1j * rng.normal(size=(N, nvec))
    return X / np.linalg.norm(X, axis=0)


@pytest.mark.parametrize("backend", ["cuda", "tc"])
@pytest.mark.parametrize("nvec", [1, 8, 16, 20, 40])
def test_hx_mos2(backend, nvec):
    ex, H = _setup("MoS2.model", 12, 2, [1., 4., 13.55])
    ex.setHxBackend(backend)
    X = _x(H.shape[0], nvec)
    Y = ex.matvec(X)
    Yo = H @ X
    assert np.abs(Y - Yo).max() / np.abs(Yo).max() < HX_TOL


@pytest.mark.parametrize("backend", ["cuda", "tc"])
def test_hx_hbn_partial_tiles(backend):
    """N = 400: not a multiple of the 128-row tile, 2N not a multiple of the 64-column tile."""
    ex, H = _setup("hBN.model", 20, 1, [1, 1, 10])
    ex.setHxBackend(backend)
    X = _x(H.shape[0], 8, seed=3)
    Y = ex.matvec(X)
    Yo = H @ X
    assert np.abs(Y - Yo).max() / np.abs(Yo).max() < HX_TOL


def test_hx_tc_matches_cuda_core_synthetic():
    from xatu_b200.synthetic import synthetic_hexagonal
    ex, H = _setup(synthetic_hexagonal(seed=1234), 24, 2, [1, 4.5, 40])
    X = _x(H.shape[0], 16, seed=5)
    ex.setHxBackend("cuda")
    Y1 = ex.matvec(X)
    ex.setHxBackend("tc")
    Y2 = ex.matvec(X)
    Yo = H @ X
    scale = np.abs(Yo).max()
    assert np.abs(Y1 - Yo).max() / scale < HX_TOL
    assert np.abs(Y2 - Yo).max() / scale < HX_TOL
    # repeated products reuse the buffers and give the same result (no stale state)
    Y3 = ex.matvec(X)
    assert np.abs(Y3 - Y2).max() / scale < 1e-6
