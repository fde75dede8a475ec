"""The large workloads pinned against the oracle (fixtures made by
tests/golden/make_large_pins.py): the oracle's energy functional at the
engine's converged FP64 density, whose commutator X^T (F P S - S P F) X
under the oracle's own integrals is below 1e-6 -- so the density is the
oracle's SCF solution and E[P] its SCF energy to second order.  The engine
must reproduce that energy to 1e-8 Ha in FP64 and 1e-6 Ha in mixed
precision, and (where the fixture holds it) the oracle's analytic gradient
at that density to 1e-7 Ha/bohr.

Cases: C30H61 STO-6G UHF, C40H82, C100H202 and the reference's rna1.xyz in
STO-3G (rscf.f90:140-156 / uscf.f90:183-198 energy expressions)."""
import glob
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
CASES = sorted(os.path.basename(p)[4:-5] for p in glob.glob(os.path.join(GOLDEN, "pin_*.json")))


def _fixture(name):
    with open(os.path.join(GOLDEN, f"pin_{name}.json")) as fh:
        return json.load(fh)


def _molecule(engine, name):
    import sys
    sys.path.insert(0, GOLDEN)
    import make_large_pins as M
    sp, xyz, basis = M.case_geometry(name)
    return engine.Molecule(sp, xyz, basis)


@pytest.mark.parametrize("precision,etol", [("fp64", 1e-8), ("mixed", 1e-6)])
@pytest.mark.parametrize("name", CASES)
def test_engine_energy_vs_oracle(engine, name, precision, etol):
    d = _fixture(name)
    mol = _molecule(engine, name)
    r = engine.run(mol, gradient="oracle_gradient_at_engine_density" in d, precision=precision, max_iter=200)
    assert r.converged and r.nbf == d["nbf"] and r.uhf == d["uhf"]
    assert abs(r.energy - d["oracle_energy_at_engine_density"]) <= etol, (r.energy,
                                                                         d["oracle_energy_at_engine_density"])
    if "oracle_gradient_at_engine_density" in d:
        g = np.array(d["oracle_gradient_at_engine_density"])
        gtol = 1e-7 if precision == "fp64" else 1e-5
        assert np.abs(r.gradient - g).max() <= gtol
