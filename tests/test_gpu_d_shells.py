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
    """Energy against the oracle's own SCF; gradient against the oracle's
    derivative integrals at the engine's converged density (1e-7), and
    against the oracle's own SCF gradient only to 1e-6: with Zn's core
    exponents the gradient moves by ~7e-8 between a DIIS error of 1e-8 and
    1e-11 in the oracle alone, so two independently converged SCFs differ
    there by a few 1e-7."""
    sp, xyz = mol()
    with engine.System(engine.Molecule(sp, xyz), max_iter=300) as s:
        r = s.scf(matrices=True)
        g = s.gradient()
    P = r.matrices["P"]
    om = oracle.molecule(sp, xyz, basis_file())
    ro = oracle.scf(om, max_iter=300)
    assert r.converged and ro.converged
    assert r.energy == pytest.approx(ro.energy, abs=1e-8)
    g_at = oracle.gradient_at_density(om, [0.5 * P, 0.5 * P], uhf=False)
    assert np.abs(g - g_at).max() < 1e-7
    assert np.abs(g - oracle.gradient(om, ro)).max() < 1e-6
    assert np.abs(g.sum(0)).max() < 1e-8


def _oracle_energy_at(oracle, om, Ds):
    """The oracle's UHF energy functional and its largest commutator
    X^T (F_s D_s S - S D_s F_s) X at the spin densities Ds."""
    S, T, V = oracle.one_electron(om)
    H = T + V
    J, K = oracle.jk(om, np.stack(Ds), 1e-12)
    Jt = J[0] + J[1]
    Fs = [H + Jt - K[0], H + Jt - K[1]]
    E = 0.5 * (np.sum((Ds[0] + Ds[1]) * H) + np.sum(Ds[0] * Fs[0]) + np.sum(Ds[1] * Fs[1])) + oracle.enuc(om)
    s, U = np.linalg.eigh(S)
    X = U / np.sqrt(s)
    comm = max(float(np.abs(X.T @ (F @ D @ S - S @ D @ F) @ X).max()) for F, D in zip(Fs, Ds))
    return E, comm


def test_d_uhf_scandium_atom_vs_oracle(engine, oracle):
    """Sc: 21 electrons, a doublet -> UHF (helper_functions.py:58-87).  An
    open-shell d atom has several UHF solutions (which d orbital the odd
    electron takes), so the engine's solution is checked against the
    oracle's own integrals: its spin densities make the oracle's UHF
    commutator vanish and give the oracle's energy functional the engine's
    energy to 1e-8 Ha."""
    import ctypes
    import torch
    from pyfacc import _native as N
    from pyfacc.distributed import _CudaView
    xyz = np.zeros((1, 3))
    with engine.System(engine.Molecule(["Sc"], xyz), max_iter=300) as s:
        r = s.scf(matrices=True)
        assert r.uhf and r.converged
        n = s.nbf
        ptr = ctypes.c_void_p()
        N.check(N.lib().pyfacc_system_density_dev(s.handle, ctypes.byref(ptr)), "density")
        Pa = torch.as_tensor(_CudaView(int(ptr.value), n * n), device="cuda").cpu().numpy().reshape(n, n).copy()
        Pt = r.matrices["P"]
    om = oracle.molecule(["Sc"], xyz, basis_file())
    E, comm = _oracle_energy_at(oracle, om, [Pa, Pt - Pa])
    assert comm < 1e-6
    assert r.energy == pytest.approx(E, abs=1e-8)


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
