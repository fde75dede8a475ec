"""The larger workloads: UHF radical in STO-6G with the analytic gradient
against central finite differences (h = 1e-4 bohr) of this engine's energy
and of the oracle's, and C100H202 in mixed precision against FP64."""
import numpy as np
import pytest

from conftest import basis_file

pytestmark = pytest.mark.gpu
H = 1e-4


def _fd(engine, species, xyz, coords, basis, **opt):
    out = {}
    for a, x in coords:
        e = []
        for s in (1, -1):
            x2 = xyz.copy()
            x2[a, x] += s * H
            e.append(engine.run(engine.Molecule(species, x2, basis), **opt).energy)
        out[(a, x)] = (e[0] - e[1]) / (2 * H)
    return out


def test_c30h61_sto6g_uhf_gradient_vs_engine_fd(engine):
    from pyfacc import geometry as G
    sp, xyz = G.radical(30, seed=2)
    mol = engine.Molecule(sp, xyz, "sto-6g")
    r = engine.run(mol, gradient=True)
    assert r.uhf and r.converged and r.nbf == 211
    coords = [(0, 0), (0, 1), (1, 2), (30, 0)]  # radical carbon, its neighbour, a hydrogen
    fd = _fd(engine, sp, xyz, coords, "sto-6g")
    for (a, x), v in fd.items():
        assert r.gradient[a, x] == pytest.approx(v, abs=5e-6), (a, x)
    assert np.abs(r.gradient.sum(0)).max() < 1e-7


def test_ethyl_radical_sto6g_vs_oracle_fd(engine, oracle):
    from pyfacc import geometry as G
    sp, xyz = G.radical(2, seed=5)
    mol = engine.Molecule(sp, xyz, "sto-6g")
    r = engine.run(mol, gradient=True)
    om = oracle.molecule(sp, xyz, basis_file("sto-6g"))
    ro = oracle.scf(om)
    assert r.energy == pytest.approx(ro.energy, abs=1e-8)
    fd = oracle.fd_gradient(sp, xyz, basis_file("sto-6g"), coords=[(0, 0), (1, 2), (3, 1)], h=H)
    for (a, x), v in fd.items():
        assert r.gradient[a, x] == pytest.approx(v, abs=2e-6), (a, x)


def test_c100h202_mixed_vs_fp64(engine):
    from pyfacc import geometry as G
    sp, xyz = G.alkane(100, seed=4)
    mol = engine.Molecule(sp, xyz, "sto-3g")
    e64 = engine.run(mol, gradient=True)
    emx = engine.run(mol, gradient=True, precision="mixed")
    assert e64.nbf == 702 and e64.converged and emx.converged
    assert abs(emx.energy - e64.energy) <= 1e-6
    assert np.abs(emx.gradient - e64.gradient).max() <= 1e-5
