"""The reference's own larger inputs (data/molecules/rna1.xyz: 131 atoms with
phosphorus, 491 basis functions; gly30.xyz: 213 atoms, 697 basis functions)
through the engine API and through the drop-in driver: SCF convergence,
mixed precision against FP64, translational invariance of the gradient."""
import ctypes

import numpy as np
import pytest

from conftest import PKG

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,nbf", [("rna1.xyz", 491), ("gly30.xyz", 697)])
def test_reference_inputs(engine, name, nbf, monkeypatch):
    import helper_functions as hf
    monkeypatch.chdir(PKG)  # ./data/molecules/<file>, as the reference's driver reads it
    n, coords, species = hf.read_xyz(name)
    mol = engine.Molecule(list(species), np.ascontiguousarray(np.asarray(coords).T), "sto-3g")
    r64 = engine.run(mol, gradient=True, max_iter=200)
    rmx = engine.run(mol, gradient=True, precision="mixed", max_iter=200)
    assert r64.nbf == nbf and r64.converged and rmx.converged
    assert abs(rmx.energy - r64.energy) <= 1e-6
    assert np.abs(rmx.gradient - r64.gradient).max() <= 1e-5
    assert np.abs(r64.gradient.sum(axis=0)).max() < 1e-7
    e = hf.run_scf(hf.load_library(), name, 1e-8, 200, ctypes.c_double(), "sto-3g")
    assert e == pytest.approx(r64.energy, abs=1e-6)
