"""Host-side derived parameters against what the reference computed."""
import os

import numpy as np
import pytest

import pyoracle as po
from ftspolysol_b200.cases import Case, Species, homopolymer
from ftspolysol_b200.derive import derive

import sys
sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
import make_golden  # noqa: E402


@pytest.mark.parametrize("idx", [0, 1, 2, 3, 4])
def test_derive_matches_reference(idx, golden_dir):
    case, _ = make_golden.golden_cases()[idx]
    g = np.load(os.path.join(golden_dir, case.name + ".npz"))
    ref = po.derived_from_golden(g)
    mine = derive(case)
    assert mine["m"] == ref["m"]
    for k in ("dV", "volume", "rho0", "a", "lB", "dt", "lambda_psi", "self_pressure"):
        assert mine[k] == pytest.approx(ref[k], rel=1e-14, abs=1e-300), k
    assert len(mine["modes"]) == len(ref["modes"])
    for a, b in zip(mine["modes"], ref["modes"]):
        assert a["coeff"] == pytest.approx(b["coeff"], rel=1e-12)
        assert a["lambda"] == b["lambda"]
        assert complex(a["gamma"]) == complex(b["gamma"])
        assert np.allclose(a["O"], b["O"], atol=1e-12)
    assert len(mine["ions"]) == len(ref["ions"])
    for a, b in zip(mine["ions"], ref["ions"]):
        assert (a["valence"], a["count"], a["smear"]) == (b["valence"], b["count"], b["smear"])
    for a, b in zip(mine["species"], ref["species"]):
        assert a["num_chains"] == b["num_chains"]
        assert a["types"] == b["types"]
        assert np.allclose(a["charges"], b["charges"])
        assert np.allclose(a["bonds"], b["bonds"])
