"""The allocation-free product xatu_hx_noalloc, called through the C ABI.

It serves callers that cannot allocate device memory themselves (codes that
keep the GPU's memory in their own pool, caller-written eigensolver loops that
cannot afford a cudaMalloc/cudaFree per product).  The test plays such a
caller: it owns every buffer (here allocated with torch) and checks the result
against the library's existing product, xatu_kernel_matvec, on two calls in a
row with different sizes, so stale scratch from the first call would show.
This file sorts last so that a run stopping at the first failure has already
run every other test; it also passes alone in a fresh process."""
import ctypes

import numpy as np
import pytest

from tests.helpers import engine_exciton, model_config

pytestmark = pytest.mark.gpu

HX_TOL = 2e-5   # same tolerance as the other H.X tests (split-BF16 planes, FP32 accumulation)


def test_noalloc_matches_existing_product_twice():
    import torch
    from xatu_b200 import _lib as L

    cfg = model_config("MoS2.model")
    ex = engine_exciton(cfg, 12, 2, [1., 4., 13.55])
    ex.BShamiltonian("mixed")
    hi, lo, dg = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
    ex._call("xatu_bse_device_buffers", ctypes.byref(hi), ctypes.byref(lo), ctypes.byref(dg))
    N = ex.excitonbasisdim
    ldk = (N + 3) // 4 * 4
    rng = np.random.default_rng(11)
    for nvec in (8, 3):
        X = rng.normal(size=(N, nvec)) + 1j * rng.normal(size=(N, nvec))
        X /= np.linalg.norm(X, axis=0)
        ref = ex.matvec(X)                       # the existing entry point
        xd = torch.from_numpy(np.ascontiguousarray(X.T)).to("cuda")   # column-major N x nvec
        yd = torch.full_like(xd, complex(np.nan, np.nan))
        stream = torch.cuda.current_stream().cuda_stream
        st = L.lib().xatu_hx_noalloc(hi, lo, dg, N, ldk, nvec, ctypes.c_void_p(xd.data_ptr()),
                                     ctypes.c_void_p(yd.data_ptr()), ctypes.c_void_p(stream))
        assert st == L.XATU_OK
        Y = yd.cpu().numpy().T
        assert np.all(np.isfinite(Y))
        assert np.abs(Y - ref).max() / np.abs(ref).max() < HX_TOL


def test_noalloc_rejects_oversize():
    from xatu_b200 import _lib as L
    import torch
    buf = torch.zeros(16, dtype=torch.complex128, device="cuda")
    p = ctypes.c_void_p(buf.data_ptr())
    assert L.lib().xatu_hx_noalloc(p, p, p, 20000, 20000, 1, p, p, None) == 6   # XATU_ERR_UNSUPPORTED
    assert L.lib().xatu_hx_noalloc(p, p, p, 16, 16, 17, p, p, None) == 6
