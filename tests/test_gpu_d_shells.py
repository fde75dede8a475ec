"""Cartesian d shells (Sc and heavier in STO-nG; basis.f90:76-82 of the
reference has no D branch) through the engine, against the oracle, which
reads them the same way: S/T/V elementwise, the ERI tensor, J/K, RHF and
UHF energies and the analytic gradient.  The d quartets run in the
warp-cooperative kernels of kernels_d.cu."""
import numpy as np
import pytest

from conftest import basis_file

pytestmark = pytest.mark.gpu
A = 1.8897259886  # angstrom -> bohr


def _zn_h2():
    return ["Zn", "H", "H"], np.array([[0.0, 0.0, 0.0], [0.05, 0.02, 1.53], [-0.03, 0.04, -1.55]]) * A


def _sc_h3():
    return ["Sc", "H", "H", "H"], np.array([[0.0, 0.0, 0.1], [1.8, 0.1, 0.0], [-0.85, 1.55, -0.05],
                                            [-0.9, -1.5, 0.05]]) * A


@pytest.mark.parametrize("boys_mode", [0, 1])
def test_d_one_electron_vs_oracle(engine, oracle, boys_mode):
    sp, xyz = _sc_h3()
    sy = engine.System(engine.Molecule(sp, xyz), boys_mode=boys_mode)
    S, T, V = (x.cpu().numpy() for x in sy.one_electron())
    om = oracle.molecule(sp, xyz, basis_file())
    So, To, Vo = oracle.one_electron(om, boys_mode=boys_mode)
    assert sy.nbf == So.shape[0] == 22
    for a, b in ((S, So), (T, To), (V, Vo)):
        assert np.abs(a - b).max() < 1e-10
    sy.close()


def test_d_eri_tensor_and_jk_vs_oracle(engine, oracle):
    import torch
    sp, xyz = _zn_h2()
    om = oracle.molecule(sp, xyz, basis_file())
    with engine.System(engine.Molecule(sp, xyz), schwarz_thresh=0.0) as s:
        n = s.nbf
        eri = s.eri_tensor().cpu().numpy()
        ref = oracle.eri_tensor(om)
        assert np.abs(eri - ref).max() < 1e-11
        rng = np.random.default_rng(4)
        D = rng.standard_normal((n, n)) * 0.2
        D = D + D.T
        J, K = s.jk(torch.tensor(D, device="cuda"))
        Jo, Ko = oracle.jk(om, D, thresh=0.0)
        assert np.abs(J.cpu().numpy() - Jo).max() < 1e-10
        assert np.abs(K.cpu().numpy() - Ko).max() < 1e-10


@pytest.mark.parametrize("mol", [_zn_h2, _sc_h3])
def test_d_rhf_energy_gradient_vs_oracle(engine, oracle, mol):
    sp, xyz = mol()
    r = engine.run(engine.Molecule(sp, xyz), gradient=True, max_iter=300)
    om = oracle.molecule(sp, xyz, basis_file())
    ro = oracle.scf(om, max_iter=300)
    go = oracle.gradient(om, ro)
    assert r.converged and ro.converged
    assert r.energy == pytest.approx(ro.energy, abs=1e-8)
    assert np.abs(r.gradient - go).max() < 1e-7
    assert np.abs(r.gradient.sum(0)).max() < 1e-8


def test_d_uhf_scandium_atom_vs_oracle(engine, oracle):
    """Sc: 21 electrons, a doublet -> UHF (helper_functions.py:58-87)."""
    xyz = np.zeros((1, 3))
    r = engine.run(engine.Molecule(["Sc"], xyz), max_iter=300)
    ro = oracle.scf(oracle.molecule(["Sc"], xyz, basis_file()), max_iter=300)
    assert r.uhf and r.converged and ro.converged
    assert r.energy == pytest.approx(ro.energy, abs=1e-8)


def test_d_mixed_precision_vs_fp64(engine):
    """The d quartets stay in FP64; the s/p quartets of the same molecule
    follow the mixed-precision rule."""
    sp, xyz = _zn_h2()
    mol = engine.Molecule(sp, xyz)
    e64 = engine.run(mol, gradient=True, max_iter=300)
    emx = engine.run(mol, gradient=True, precision="mixed", max_iter=300)
    assert emx.converged
    assert abs(emx.energy - e64.energy) <= 1e-6
    assert np.abs(emx.gradient - e64.gradient).max() <= 1e-5
