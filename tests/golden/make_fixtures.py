"""Regenerate the committed test fixtures from a checkout of the reference.

    python tests/golden/make_fixtures.py /path/to/xatu

Copies the reference's example inputs used by its own regression tests
(examples/material_models/{hBN,hBN_spinful,MoS2}.model and
test/data/hBN_spinless.txt) and extracts the golden values of the BSE hot
path from test/tests.cpp into reference_goldens.json.  Every value is checked
against the text of tests.cpp, so a fixture cannot drift from its source.
"""
import json
import os
import re
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))

# (name, tests.cpp line range, model, ncell, nbands, params, extra, nstates, expected [(E, deg)], tol)
CASES = [
    ("hBN_fulldiag", "150-180", "hBN.model", 20, 1, [1, 1, 10], {}, 3, [[5.335690, 2], [6.074062, 1]], 1e-4),
    ("hBN_davidson", "182-212", "hBN.model", 20, 1, [1, 1, 10], {"method": "davidson"}, 3,
     [[5.335690, 2], [6.074062, 1]], 1e-4),
    ("hBN_lanczos", "214-244", "hBN.model", 20, 1, [1, 1, 10], {"method": "sparse"}, 3,
     [[5.335690, 2], [6.074062, 1]], 1e-4),
    ("hBN_reciprocal", "246-279", "hBN.model", 20, 1, [1, 1, 10], {"mode": "reciprocalspace", "nG": 5}, 3,
     [[6.234291, 1], [6.236636, 1], [6.731819, 1]], 1e-4),
    ("hBN_spinful", "401-431", "hBN_spinful.model", 20, 2, [1, 1, 10], {}, 12, [[5.335690, 8], [6.074062, 4]], 1e-4),
    ("MoS2_energies", "547-577", "MoS2.model", 12, 2, [1., 4., 13.55], {}, 2, [[1.768783, 2], [1.780562, 2]], 1e-4),
    ("MoS2_Q_m0.1", "660-702", "MoS2.model", 12, 2, [1., 4., 13.55], {"Q": [0, -0.1, 0]}, 2, [[1.810464, 2]], 1e-5),
    ("MoS2_Q_m0.05", "660-702", "MoS2.model", 12, 2, [1., 4., 13.55], {"Q": [0, -0.05, 0]}, 2, [[1.780106, 2]], 1e-5),
    ("MoS2_Q_0", "660-702", "MoS2.model", 12, 2, [1., 4., 13.55], {"Q": [0, 0.0, 0]}, 2, [[1.768783, 2]], 1e-5),
    ("MoS2_Q_0.05", "660-702", "MoS2.model", 12, 2, [1., 4., 13.55], {"Q": [0, 0.05, 0]}, 2, [[1.780106, 2]], 1e-5),
    ("MoS2_Q_0.1", "660-702", "MoS2.model", 12, 2, [1., 4., 13.55], {"Q": [0, 0.1, 0]}, 2, [[1.810464, 2]], 1e-5),
    ("MoS2_exchange", "704-737", "MoS2.model", 12, 2, [1., 4., 13.55], {"Q": [0, 0.1, 0], "exchange": True}, 4,
     [[1.810464, 2], [1.825740, 1], [1.855544, 1]], 1e-5),
    ("MoS2_reducedBZ", "739-774", "MoS2.model", 12, 2, [1., 4., 13.55],
     {"factor": 2, "shift": [0.6628, -1.1480, 0]}, 4,
     [[1.795378, 1], [1.809810, 1], [1.935880, 1], [1.950567, 1]], 1e-4),
]

HASHES = {
    # tests.cpp:19-61 (model parsing), :125-148 (exciton file parsing)
    "model_parsing": {"file": "hBN.model", "filling": 1, "ndim": 2, "orbitals": [1, 1],
                      "bravais_hash": [4.55422, 2.05422], "motif_hash": [0, 3.90211],
                      "bravais_vectors_hash": [0, -0.110843, 2.38916, 2.05422, 4.55422],
                      "hamiltonian_hash": [-1.34375, -0.9, -0.9, -0.0375, -0.0375], "tol": 1e-4},
    "exciton_parsing": {"file": "hBN_spinless.txt", "label": "hBN_N30", "ncell": 30, "nbands": 1,
                        "dielectric": [1, 1, 10]},
    # tests.cpp:281-321, :579-619 (k-space wavefunction hashes of the lowest 2 states)
    "hBN_kwf": {"model": "hBN.model", "ncell": 20, "nbands": 1, "params": [1, 1, 10], "nstates": 2,
                "hash": 1.086145105, "tol": 1e-5},
    "MoS2_kwf": {"model": "MoS2.model", "ncell": 12, "nbands": 2, "params": [1., 4., 13.55], "nstates": 2,
                 "hash": 1.1814790902, "tol": 1e-5},
    # tests.cpp:323-369 (real-space wavefunction hash: hole on atom 1 of cell 0, electron cells within
    # |a1| * ncell, summed over the lowest 2 states)
    "hBN_rswf": {"model": "hBN.model", "ncell": 20, "nbands": 1, "params": [1, 1, 10], "nstates": 2,
                 "hole_index": 1, "hole_cell": [0, 0, 0], "radius_cells": 20, "hash": 3.4185866144, "tol": 1e-5},
    # tests.cpp:432-462 (spinX of the lowest 4 states of spinful hBN: total Sz, |hole| = |electron| = 1/2)
    "hBN_spin": {"model": "hBN_spinful.model", "ncell": 16, "nbands": 2, "params": [1, 1, 10], "nstates": 4,
                 "total": [-1, 0, 0, 1], "abs_parts": 0.5, "tol": 1e-2},
}


def _check_against_tests(ref: str):
    text = open(os.path.join(ref, "test", "tests.cpp")).read()
    for case in CASES:
        for e, d in case[8]:
            if f"{e:.6f}" not in text:
                raise SystemExit(f"{case[0]}: {e:.6f} not found in tests.cpp")
    for key in ("hBN_kwf", "MoS2_kwf", "hBN_rswf"):
        if repr(HASHES[key]["hash"]) not in text:
            raise SystemExit(f"{key}: hash not found in tests.cpp")
    for v in ("4.55422", "3.90211", "-0.110843", "-1.34375", "-0.0375"):
        if v not in text:
            raise SystemExit(f"parse hash {v} not found")
    if "arma::vec{-1, 0, 0, 1}" not in text or "WithinAbs(0.5, 1E-2)" not in text:
        raise SystemExit("spin golden not found")
    if not re.search(r"expectedName = \"hBN_N30\"", text):
        raise SystemExit("exciton parse golden not found")


def main(ref: str):
    _check_against_tests(ref)
    os.makedirs(os.path.join(HERE, "models"), exist_ok=True)
    for m in ("hBN.model", "hBN_spinful.model", "MoS2.model"):
        shutil.copyfile(os.path.join(ref, "examples", "material_models", m), os.path.join(HERE, "models", m))
    shutil.copyfile(os.path.join(ref, "test", "data", "hBN_spinless.txt"), os.path.join(HERE, "hBN_spinless.txt"))
    out = {"source": "xatu v1.3.1 test/tests.cpp", "cases": [], "hashes": HASHES}
    for name, lines, model, ncell, nbands, params, extra, nstates, expected, tol in CASES:
        out["cases"].append({"name": name, "tests_cpp_lines": lines, "model": model, "ncell": ncell,
                             "nbands": nbands, "params": params, "extra": extra, "nstates": nstates,
                             "expected": expected, "tol": tol})
    with open(os.path.join(HERE, "reference_goldens.json"), "w") as fh:
        json.dump(out, fh, indent=1)
    print("fixtures written")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit("usage: python tests/golden/make_fixtures.py <path of the xatu source tree>")
    main(sys.argv[1])
