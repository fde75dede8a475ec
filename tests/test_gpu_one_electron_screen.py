"""The engine's one-electron pair screen on the GPU (System::upload_shells
leaves out shell pairs on two atoms whose primitive prefactors are all below
1e-25): the engine's S, T and V, with the screen active, against the
oracle's unscreened matrices elementwise, on a 40-carbon chain (most
two-atom pairs screened) and on the reference's rna1.xyz (P atoms, whose
larger exponents and nuclear charges test the margin of the bound)."""
import os

import numpy as np
import pytest

from conftest import basis_file

pytestmark = pytest.mark.gpu
PKG = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "pyfacc-scf_b200")


def _case(engine, name):
    if name == "c40h82":
        from pyfacc import geometry as G
        return G.alkane(40, seed=40)
    m = engine.Molecule.from_xyz(os.path.join(PKG, "data", "molecules", "rna1.xyz"), "sto-3g")
    return list(m.species), np.asarray(m.coords)


@pytest.mark.parametrize("name", ["c40h82", "rna1"])
def test_screened_one_electron_matrices_vs_oracle(engine, oracle, name):
    sp, xyz = _case(engine, name)
    with engine.System(engine.Molecule(sp, xyz, "sto-3g")) as s:
        S, T, V = (x.cpu().numpy() for x in s.one_electron())
    om = oracle.molecule(sp, xyz, basis_file("sto-3g"))
    So, To, Vo = oracle.one_electron(om)
    assert S.shape == So.shape
    for a, b in ((S, So), (T, To), (V, Vo)):
        assert np.abs(a - b).max() < 1e-10
    if name == "c40h82":  # the screen does act: entries of distant pairs are exactly zero
        assert (S == 0.0).sum() > 0.2 * S.size
