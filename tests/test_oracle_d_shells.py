"""d shells in the oracle (ground work for l = 2 classes of the engine; the
reference's parser has no D branch, basis.f90:76-82, and the engine
rejects them with PYFACC_ERR_UNSUPPORTED_L).  Cartesian d components in the
order xx, xy, xz, yy, yz, zz, each normalised on its own.  Checked with
unit self-overlaps, two independent ERI formulations (OS/HGP with
per-component normalisation against Cook/THO), and the analytic gradient
against central finite differences."""
import os

import numpy as np
import pytest

from conftest import basis_file

H_SP_D = """****
H     0
S   3   1.00
      3.42525091             0.15432897
      0.62391373             0.53532814
      0.16885540             0.44463454
P   1   1.00
      0.75                   1.00000000
D   2   1.00
      1.10                   0.60000000
      0.35                   0.50000000
****
"""

D_ONLY = """****
He     0
D   1   1.00
      0.90                   1.00000000
****
"""


def _write(tmp_path, text):
    p = os.path.join(str(tmp_path), "basis.txt")
    with open(p, "w") as fh:
        fh.write(text)
    return p


def test_d_components_have_unit_self_overlap(oracle, tmp_path):
    mol = oracle.molecule(["He"], np.zeros((1, 3)), _write(tmp_path, D_ONLY), nalpha=1, nbeta=1)
    assert list(mol.shells.l) == [2] and mol.shells.nbf == 6
    S, T, V = oracle.one_electron(mol)
    assert np.allclose(np.diag(S), 1.0, atol=1e-13)
    # off-diagonal: <xx|yy> = 1/3 for one normalised primitive, <xx|xy> = 0
    assert S[0, 3] == pytest.approx(1.0 / 3.0, abs=1e-13)
    assert abs(S[0, 1]) < 1e-14


def test_d_shell_eri_formulations_agree(oracle, tmp_path):
    xyz = np.array([[0.0, 0.0, 0.0], [0.3, -0.2, 1.4], [1.1, 0.9, -0.4]])
    mol = oracle.molecule(["H", "H", "H"], xyz, _write(tmp_path, H_SP_D), nalpha=2, nbeta=1)
    l = list(mol.shells.l)
    d = [i for i, x in enumerate(l) if x == 2]
    p = [i for i, x in enumerate(l) if x == 1]
    s = [i for i, x in enumerate(l) if x == 0]
    quartets = [(d[0], d[1], d[2], d[0]), (d[1], s[0], p[2], d[2]), (p[0], d[2], s[1], s[2]),
                (d[0], d[0], d[0], d[0]), (s[0], s[1], d[2], p[1])]
    for q in quartets:
        os_ = np.array(oracle.eri_quartet(mol, *q, method=0))
        cook = np.array(oracle.eri_quartet(mol, *q, method=1))
        assert np.abs(os_ - cook).max() <= 1e-12 * max(1.0, np.abs(cook).max()), q


def test_d_shell_gradient_vs_finite_differences(oracle, tmp_path):
    bf = _write(tmp_path, H_SP_D)
    sp = ["H", "H"]
    xyz = np.array([[0.0, 0.0, 0.0], [0.2, -0.1, 1.45]])
    mol = oracle.molecule(sp, xyz, bf)
    res = oracle.scf(mol)
    g = oracle.gradient(mol, res)
    assert np.abs(g.sum(0)).max() < 1e-10
    fd = oracle.fd_gradient(sp, xyz, bf, coords=[(1, 0), (1, 2)], h=1e-4)
    for (a, x), v in fd.items():
        assert g[a, x] == pytest.approx(v, abs=2e-7), (a, x)
