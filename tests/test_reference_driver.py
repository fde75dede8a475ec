"""The drop-in driver passes run_scf_c exactly what the reference's own
driver passes (golden vectors recorded from PyFAcc-SCF's
src/python/helper_functions.py by tests/golden/make_reference_args.py):
species bytes, coordinates bit for bit in memory order, electron counts,
z_num, and the same spin assignments and errors."""
import ctypes
import json
import os
import struct
import sys

import numpy as np
import pytest

from conftest import PKG

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "reference_driver_args.json")


class Recorder:
    def __init__(self):
        self.calls = []

    def run_scf_c(self, natoms, nelectrons, charge, nalpha, nbeta, species, coords, eps, max_iter, energy, basis,
                  z_num):
        n = natoms.value
        self.calls.append({
            "natoms": n, "nelectrons": nelectrons.value, "charge": charge.value, "nalpha": nalpha.value,
            "nbeta": nbeta.value, "species": bytes(species).decode("ascii"),
            "coords_hex": [struct.pack("<d", coords[i]).hex() for i in range(3 * n)], "eps_scf": eps.value,
            "max_iter": max_iter.value, "basis": basis.decode(), "z_num": [z_num[i] for i in range(n)]})


@pytest.fixture(scope="module")
def golden():
    with open(GOLDEN) as fh:
        return json.load(fh)


@pytest.fixture(scope="module")
def helpers():
    sys.path.insert(0, PKG)
    import helper_functions as H
    return H


def test_run_scf_c_arguments_match_reference(golden, helpers, monkeypatch):
    monkeypatch.chdir(PKG)  # read_xyz opens ./data/molecules/<file>, as the reference does
    assert len(golden["calls"]) >= 10
    for f, want in golden["calls"].items():
        rec = Recorder()
        helpers.run_scf(rec, f, 1e-10, 10, ctypes.c_double(), "sto-3g")
        assert rec.calls[0] == want, f


def test_spin_electrons_match_reference(golden, helpers):
    for key, want in golden["spin"].items():
        sp, charge = key.split("/")
        species = np.array(sp.split(","))
        if isinstance(want, dict):
            with pytest.raises(ValueError):
                helpers.compute_spin_electrons(species, int(charge))
        else:
            assert list(helpers.compute_spin_electrons(species, int(charge))) == want, key
