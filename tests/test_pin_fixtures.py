"""The large-workload pin fixtures (tests/golden/pin_*.json, made by
tests/golden/make_large_pins.py) are what they claim: the density they were
made from is an SCF solution under the oracle's own integrals (commutator
X^T (F P S - S P F) X below 1e-6) with the right electron counts
(tr P S = 2 n_occ for RHF, n_alpha and n_beta for UHF), and its oracle
energy agrees with the engine's energy at the time of the dump."""
import glob
import json
import os

import pytest

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
FILES = sorted(glob.glob(os.path.join(GOLDEN, "pin_*.json")))


@pytest.mark.parametrize("path", FILES, ids=[os.path.basename(p) for p in FILES])
def test_pin_fixture_is_an_oracle_scf_solution(path):
    with open(path) as fh:
        d = json.load(fh)
    assert d["oracle_commutator_max"] < 1e-6
    factor = 1 if d["uhf"] else 2
    for tr, occ in zip(d["electron_count_tr_PS"], d["occupations"]):
        assert abs(tr - factor * occ) < 1e-8
    assert abs(d["oracle_energy_at_engine_density"] - d["engine_fp64_energy_at_dump"]) < 1e-8
