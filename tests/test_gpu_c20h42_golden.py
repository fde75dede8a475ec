"""The C20H42/STO-3G benchmark molecule (142 basis functions) against the
oracle's converged energy and analytic gradient, stored as a fixture
(tests/golden/make_golden.py c20h42): FP64 to 1e-8 Ha and 1e-7 Ha/bohr,
mixed precision to 1e-6 Ha and 1e-5 Ha/bohr."""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "c20h42_sto3g.json")


@pytest.fixture(scope="module")
def golden():
    with open(GOLDEN) as fh:
        return json.load(fh)


@pytest.mark.parametrize("precision,etol,gtol", [("fp64", 1e-8, 1e-7), ("mixed", 1e-6, 1e-5)])
def test_c20h42_vs_oracle(engine, golden, precision, etol, gtol):
    from pyfacc import geometry as G
    mol = engine.Molecule(*G.alkane(20, seed=1), "sto-3g")
    r = engine.run(mol, gradient=True, precision=precision)
    assert r.converged and r.nbf == golden["nbf"] == 142
    assert abs(r.energy - golden["energy"]) <= etol
    assert np.abs(r.gradient - np.array(golden["gradient"])).max() <= gtol
