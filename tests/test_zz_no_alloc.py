"""The allocation-free product xatu_hx_noalloc, called through the C ABI.

It serves callers that cannot allocate device memory themselves (codes that
keep the GPU's memory in their own pool, caller-written eigensolver loops that
cannot afford a cudaMalloc/cudaFree per product).  The test plays such a
caller: it owns every buffer (here allocated with torch) and checks the result
against the library's existing product, xatu_kernel_matvec, and against the
oracle's FP64 matrix times x, on calls in a row with different sizes, so stale
scratch from an earlier call would show.  nvec 8 and 3 use the 16-row operand
layout, nvec 13 the 32-row one.  This file sorts last so that a run stopping
at the first failure has already run every other test; it also passes alone in
a fresh process."""
import ctypes

import numpy as np
import pytest

from tests.helpers import engine_exciton, model_config, oracle_exciton

pytestmark = pytest.mark.gpu

HX_TOL = 2e-5   # same tolerance as the other H.X tests (split-BF16 planes, FP32 accumulation)


def _noalloc(L, hi, lo, dg, N, ldk, X, stream=None):
    import torch
    nvec = X.shape[1]
    xd = torch.from_numpy(np.ascontiguousarray(X.T)).to("cuda")   # column-major N x nvec
    yd = torch.full_like(xd, complex(np.nan, np.nan))
    if stream is None:
        stream = torch.cuda.current_stream().cuda_stream
    st = L.lib().xatu_hx_noalloc(hi, lo, dg, N, ldk, nvec, ctypes.c_void_p(xd.data_ptr()),
                                 ctypes.c_void_p(yd.data_ptr()), ctypes.c_void_p(stream))
    return st, yd.cpu().numpy().T


def test_noalloc_matches_existing_product_and_oracle():
    from xatu_b200 import _lib as L

    cfg = model_config("MoS2.model")
    kw = dict(Q=(0, 0.1, 0), exchange=True)
    ex = engine_exciton(cfg, 12, 2, [1., 4., 13.55], **kw)
    orc = oracle_exciton(cfg, 12, 2, [1., 4., 13.55], **kw)
    ex.upload_bands(orc.eigval, orc.eigvec, orc.eigvalQ, orc.eigvecQ)
    ex.BShamiltonian("mixed")
    Ho = orc.bs_hamiltonian()
    hi, lo, dg = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
    ex._call("xatu_bse_device_buffers", ctypes.byref(hi), ctypes.byref(lo), ctypes.byref(dg))
    N = ex.excitonbasisdim
    ldk = (N + 3) // 4 * 4
    rng = np.random.default_rng(11)
    for nvec in (8, 3, 13, 13):
        X = rng.normal(size=(N, nvec)) + 1j * rng.normal(size=(N, nvec))
        X /= np.linalg.norm(X, axis=0)
        ref = ex.matvec(X)                       # the existing entry point
        st, Y = _noalloc(L, hi, lo, dg, N, ldk, X)
        assert st == L.XATU_OK
        assert np.all(np.isfinite(Y))
        assert np.abs(Y - ref).max() / np.abs(ref).max() < HX_TOL
        Yo = Ho @ X                              # the oracle's FP64 matrix
        assert np.abs(Y - Yo).max() / np.abs(Yo).max() < HX_TOL


def test_noalloc_rejects_oversize_and_capture():
    import torch
    from xatu_b200 import _lib as L
    buf = torch.zeros(16, dtype=torch.complex128, device="cuda")
    p = ctypes.c_void_p(buf.data_ptr())
    assert L.lib().xatu_hx_noalloc(p, p, p, 20000, 20000, 1, p, p, None) == 6   # XATU_ERR_UNSUPPORTED
    assert L.lib().xatu_hx_noalloc(p, p, p, 16, 16, 17, p, p, None) == 6
    # on a capturing stream the call returns XATU_ERR_STATE before it touches the stream
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(s):
        g.capture_begin()
        st = L.lib().xatu_hx_noalloc(p, p, p, 16, 16, 1, p, p, ctypes.c_void_p(s.cuda_stream))
        buf.add_(1)
        g.capture_end()
    assert st == 4   # XATU_ERR_STATE
