"""The benchmark molecules against the oracle's converged energy and
analytic gradient, stored as fixtures (tests/golden/make_golden.py c20h42 |
c40h82): C20H42/STO-3G (142 basis functions) and the north-star molecule
C40H82/STO-3G (282 basis functions); FP64 to 1e-8 Ha and 1e-7 Ha/bohr,
mixed precision to 1e-6 Ha and 1e-5 Ha/bohr."""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
CASES = {"c20h42": (20, 1, 142), "c40h82": (40, 40, 282)}


def _golden(name):
    with open(os.path.join(GOLDEN, f"{name}_sto3g.json")) as fh:
        return json.load(fh)


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("precision,etol,gtol", [("fp64", 1e-8, 1e-7), ("mixed", 1e-6, 1e-5)])
def test_alkane_vs_oracle(engine, name, precision, etol, gtol):
    from pyfacc import geometry as G
    n, seed, nbf = CASES[name]
    golden = _golden(name)
    mol = engine.Molecule(*G.alkane(n, seed=seed), "sto-3g")
    r = engine.run(mol, gradient=True, precision=precision)
    assert r.converged and r.nbf == golden["nbf"] == nbf
    assert abs(r.energy - golden["energy"]) <= etol
    assert np.abs(r.gradient - np.array(golden["gradient"])).max() <= gtol
