"""The drop-in helper_functions restate the reference's Python driver."""
import os

import numpy as np
import pytest

from conftest import MOL_DIR


def test_read_xyz_layout_is_atom_major(oracle):
    import helper_functions as hf
    n, c, s = hf.read_xyz("h2o.xyz")
    n2, c2, s2 = oracle.read_xyz(os.path.join(MOL_DIR, "h2o.xyz"))
    assert n == 3 and list(s) == ["O", "H", "H"]
    assert np.allclose(c, c2)
    # memory order handed to run_scf_c: x1 y1 z1 x2 ...
    flat = np.frombuffer(np.array(c, dtype=np.float64).tobytes(order="A"), dtype=np.float64)
    assert np.allclose(flat, c.T.reshape(-1))


def test_spin_and_multiplicity_rules():
    import helper_functions as hf
    assert hf.compute_spin_electrons(["O", "H", "H"]) == (5, 5, 1)
    assert hf.compute_spin_electrons(["O", "O"]) == (9, 7, 3)      # known exception O2 -> triplet
    assert hf.compute_spin_electrons(["O", "H"]) == (5, 4, 2)
    assert hf.guess_multiplicity(["N", "N"]) == 4
    # 14 electrons cannot be a quartet: the reference raises (helper_functions.py:82-83)
    with pytest.raises(ValueError):
        hf.compute_spin_electrons(["N", "N"])


def test_invalid_xyz_line_raises(tmp_path, monkeypatch):
    import helper_functions as hf
    d = tmp_path / "data" / "molecules"
    d.mkdir(parents=True)
    (d / "bad.xyz").write_text("2\n\nH 0 0 0\nH 0 0\n")
    monkeypatch.chdir(tmp_path)
    with pytest.raises(ValueError):
        hf.read_xyz("bad.xyz")


def test_geometry_builders():
    from pyfacc import geometry as G
    sp, x = G.alkane(20, 1)
    assert sp.count("C") == 20 and sp.count("H") == 42
    sp, x = G.radical(30, 2)
    assert sp.count("C") == 30 and sp.count("H") == 61
    cl = G.water_clusters(8, seed=3)
    for s, xyz in cl:
        n = len(s) // 3
        assert 4 <= n <= 16
        O = xyz[0::3] / G.ANG
        d = np.linalg.norm(O[:, None] - O[None], axis=-1) + np.eye(n) * 10
        assert d.min() >= 2.7 - 1e-9
