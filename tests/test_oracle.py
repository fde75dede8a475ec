"""The oracle itself: pinned against closed forms, mpmath, an independent
ERI formulation, brute-force J/K, textbook energies and finite differences."""
import json
import os

import numpy as np
import pytest

from conftest import basis_file, MOL_DIR

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_boys_accurate_vs_mpmath_fixture(oracle):
    ref = json.load(open(os.path.join(GOLDEN, "boys_mpmath.json")))
    for m, x, v in ref["values"]:
        assert oracle.boys(m, x) == pytest.approx(v, rel=2e-15, abs=1e-300)


def test_boys_trapezoid_is_the_reference_rule(oracle):
    # boys.f90:9-43 -- small-x Taylor branch and the 1001-point trapezoid
    assert oracle.boys(2, 1e-7, 1) == pytest.approx(1 / 5 - 1e-7 / 7, rel=1e-15)
    x, nu = 2.5, 1
    t = np.linspace(0.0, 1.0, 1001)
    f = t ** (2 * nu) * np.exp(-x * t * t)
    trap = (f.sum() - 0.5 * (f[0] + f[-1])) / 1000
    assert oracle.boys(nu, x, 1) == pytest.approx(trap, rel=1e-13)


def _h2o(oracle, basis="sto-3g"):
    n, c, s = oracle.read_xyz(os.path.join(MOL_DIR, "h2o.xyz"))
    return oracle.molecule(s, c.T, basis_file(basis))


def test_shell_order_follows_basis_file(oracle):
    mol = _h2o(oracle)
    # H section precedes O in sto-3g.txt: [H1 s, H2 s, O 1s, O 2s, O 2p]
    assert list(mol.shells.l) == [0, 0, 0, 0, 1]
    assert list(mol.shells.atom) == [1, 2, 0, 0, 0]
    assert mol.shells.nbf == 7


def test_os_and_cook_eri_agree(oracle):
    mol = oracle.molecule(["O", "H", "H", "C"], np.array([[0, 0, 0], [0, 1.4, 1.1], [0, -1.5, 1.0], [2.1, 0.3, -1.2]]),
                          basis_file("sto-3g"))
    ns = len(mol.shells.l)
    rng = np.random.default_rng(5)
    for _ in range(30):
        a, b, c, d = rng.integers(0, ns, 4)
        o1 = oracle.eri_quartet(mol, a, b, c, d, method=0)
        o2 = oracle.eri_quartet(mol, a, b, c, d, method=1)
        assert np.max(np.abs(o1 - o2)) < 1e-12


def test_ssss_closed_form(oracle):
    # two normalised s primitives on each of two centres: (ss|ss) = 2 pi^2.5/(pq sqrt(p+q)) e^... F0
    import math
    a, b, c, d = 0.8, 1.3, 0.5, 2.0
    A, B, C, D = np.zeros(3), np.array([0, 0, 1.0]), np.array([1.0, 0, 0]), np.array([1.0, 1.0, 0])
    p, q = a + b, c + d
    P, Q = (a * A + b * B) / p, (c * C + d * D) / q
    rho = p * q / (p + q)
    T = rho * np.sum((P - Q) ** 2)
    F0 = 0.5 * math.sqrt(math.pi / T) * math.erf(math.sqrt(T))
    N = lambda x: (2 * x / math.pi) ** 0.75
    ref = (2 * math.pi ** 2.5 / (p * q * math.sqrt(p + q)) * math.exp(-a * b / p * np.sum((A - B) ** 2))
           * math.exp(-c * d / q * np.sum((C - D) ** 2)) * F0 * N(a) * N(b) * N(c) * N(d))
    from oracle import Shells
    sh = Shells(l=np.zeros(4, np.int32), atom=np.arange(4, dtype=np.int32),
                center=np.ascontiguousarray(np.array([A, B, C, D])), poff=np.arange(5, dtype=np.int32),
                exps=np.array([a, b, c, d]), coefs=np.ones(4))
    sh.bf_off = np.arange(5, dtype=np.int32)
    sh.nbf = 4
    mol = oracle.Molecule(["H"] * 4, np.ones(4, np.int32), np.array([A, B, C, D]), 2, 2, sh)
    v = oracle.eri_quartet(mol, 0, 1, 2, 3)[0, 0, 0, 0]
    assert v == pytest.approx(ref, rel=1e-13)


def test_jk_matches_brute_force(oracle):
    mol = _h2o(oracle)
    T = oracle.eri_tensor(mol)
    assert np.abs(T - T.transpose(1, 0, 2, 3)).max() < 1e-14
    assert np.abs(T - T.transpose(2, 3, 0, 1)).max() < 1e-14
    rng = np.random.default_rng(0)
    D = rng.standard_normal((7, 7))
    D = D + D.T
    J, K = oracle.jk(mol, D, thresh=0)
    assert np.abs(J - np.einsum('mnls,ls->mn', T, D)).max() < 1e-13
    assert np.abs(K - np.einsum('mlns,ls->mn', T, D)).max() < 1e-13


def test_textbook_energies(oracle):
    # H2O / STO-3G at the Crawford-project geometry: -74.942079928 Ha with
    # renormalised contractions; the reference does not renormalise, which
    # moves the energy by ~3e-8.
    xyz = np.array([[0.0, -0.143225816552, 0.0], [1.638036840407, 1.136548822547, 0.0],
                    [-1.638036840407, 1.136548822547, 0.0]])
    mol = oracle.molecule(["O", "H", "H"], xyz, basis_file())
    assert oracle.scf(mol).energy == pytest.approx(-74.942079928, abs=1e-7)
    h = oracle.molecule(["H"], np.zeros((1, 3)), basis_file())
    S, T, V = oracle.one_electron(h)
    assert (T + V)[0, 0] == pytest.approx(-0.466581850, abs=2e-9)
    h2 = oracle.molecule(["H", "H"], np.array([[0, 0, 0], [0, 0, 1.4]]), basis_file())
    assert oracle.scf(h2).energy == pytest.approx(-1.1167143, abs=1e-6)


def test_h2o_energy_fixture(oracle):
    ref = json.load(open(os.path.join(GOLDEN, "h2o_sto3g.json")))
    mol = _h2o(oracle)
    r = oracle.scf(mol)
    assert r.converged
    assert r.energy == pytest.approx(ref["energy"], abs=1e-10)
    S, T, V = oracle.one_electron(mol, boys_mode=1)
    assert np.abs(V - np.array(ref["V_trapezoid"])).max() < 1e-12


def test_gradient_matches_finite_differences(oracle):
    n, c, s = oracle.read_xyz(os.path.join(MOL_DIR, "h2o.xyz"))
    mol = oracle.molecule(s, c.T, basis_file())
    r = oracle.scf(mol)
    g = oracle.gradient(mol, r)
    fd = oracle.fd_gradient(s, c.T, basis_file(), coords=[(0, 2), (1, 1), (2, 2)])
    for (a, x), v in fd.items():
        assert g[a, x] == pytest.approx(v, abs=1e-7)
    assert np.abs(g.sum(0)).max() < 1e-10


def test_uhf_doublet_and_rhf_equals_uhf(oracle):
    mol = oracle.molecule(["O", "H"], np.array([[0, 0, 0], [0, 0, 1.83]]), basis_file())
    assert (mol.nalpha, mol.nbeta) == (5, 4)
    r = oracle.scf(mol)
    assert r.uhf and r.converged
    h2o = _h2o(oracle)
    assert oracle.scf(h2o, uhf=True).energy == pytest.approx(oracle.scf(h2o).energy, abs=1e-9)
