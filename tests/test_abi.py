"""The C-ABI library: loads without a GPU, exports every declared symbol, and
its host-only geometry helpers match the oracle's restatement of Lattice.cpp."""
import os
import re

import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import model_config
from xatu_b200 import _lib as L

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "xatu_bse.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(xatu_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = L.lib()
    names = declared_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(L.EXPORTED_SYMBOLS)
    assert lib.xatu_abi_version() == 1


@pytest.mark.parametrize("model,n", [("hBN.model", 20), ("hBN.model", 7), ("MoS2.model", 12), ("MoS2.model", 9)])
def test_mesh_and_supercell_match_oracle(model, n):
    si = model_config(model).systemInfo
    rec = L.reciprocal_lattice(si.ndim, si.bravaisLattice)
    assert np.allclose(rec, O.reciprocal_lattice(si.bravaisLattice, si.ndim), rtol=0, atol=1e-13)
    k = L.mesh_mp(si.ndim, rec, n)
    assert np.allclose(k, O.brillouin_zone_mesh(rec, si.ndim, n), rtol=0, atol=1e-13)
    for factor in (1, 2, 3):
        kr = L.mesh_reduced(si.ndim, rec, n, factor)
        assert np.allclose(kr, O.reduced_brillouin_zone_mesh(rec, si.ndim, n, factor)[0], rtol=0, atol=1e-13)
    a = np.linalg.norm(si.bravaisLattice[0])
    for cut in (n / 2.5, 2.0, n):
        c = L.truncate_supercell(si.ndim, si.bravaisLattice, n, a * cut)
        co = O.truncate_supercell(si.bravaisLattice, si.ndim, n, a * cut)
        assert c.shape == co.shape
        assert np.allclose(c, co, rtol=0, atol=1e-12)


@pytest.mark.parametrize("n,factor", [(6, 1), (7, 1), (12, 1), (5, 2), (6, 3)])
def test_equivalent_point_exhaustive(n, factor):
    """findEquivalentPointBZ for every k' - k of the (sub)mesh, even and odd n, factor > 1."""
    si = model_config("hBN.model").systemInfo
    rec = O.reciprocal_lattice(si.bravaisLattice, si.ndim)
    inv = O.inverse_reciprocal_matrix(rec)
    if factor == 1:
        k = O.brillouin_zone_mesh(rec, 2, n)
    else:
        k, _ = O.reduced_brillouin_zone_mesh(rec, 2, n, factor)
        k = k + np.array([0.31, -0.2, 0])
    diffs = (k[None, :, :] - k[:, None, :]).reshape(-1, 3)
    got = L.equivalent_points(2, rec, n * factor, diffs)
    want = np.array([O.find_equivalent_point(rec, inv, n * factor, d) for d in diffs])
    assert np.array_equal(got, want)
    assert got.min() >= 0 and got.max() < (n * factor) ** 2
    # the mapped mesh point equals k' - k modulo a reciprocal lattice vector
    mesh = O.brillouin_zone_mesh(rec, 2, n * factor)
    red = (diffs - mesh[got]) @ np.linalg.pinv(rec)
    assert np.allclose(red, np.round(red), atol=1e-9)


def test_status_codes_without_gpu_calls():
    lib = L.lib()
    with pytest.raises(L.XatuError):
        L.check(lib.xatu_mesh_mp(0, None, 4, None))
    with pytest.raises(L.XatuError):
        L.check(lib.xatu_truncate_supercell(2, None, 4, 1.0, None, None))
