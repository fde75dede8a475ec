"""GPU parity: the sm_100a kernels against the CPU oracle on the same inputs.

Tolerances: one-electron matrices elementwise 1e-10 (either Boys mode), ERIs
1e-12 absolute, J/K 1e-10, energies 1e-8 Ha, analytic gradient 1e-7 Ha/bohr
against the oracle's analytic gradient, mixed precision |dE| <= 1e-6 Ha.
"""
import ctypes
import json
import os

import numpy as np
import pytest

from conftest import MOL_DIR, basis_file

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _pair(engine, oracle, species, xyz, basis="sto-3g"):
    xyz = np.asarray(xyz, dtype=np.float64).reshape(-1, 3)
    return engine.Molecule(species, xyz, basis), oracle.molecule(species, xyz, basis_file(basis))


def _h2o(engine, oracle, basis="sto-3g"):
    n, c, s = oracle.read_xyz(os.path.join(MOL_DIR, "h2o.xyz"))
    return _pair(engine, oracle, list(s), c.T, basis)


MOLS = {
    "h2o": None,
    "ch2o": (["C", "O", "H", "H"], [[0, 0, 0], [0, 0, 2.28], [0, 1.77, -1.1], [0, -1.77, -1.1]]),
    "nh3_co": (["N", "H", "H", "H", "C", "O"], [[0, 0, 0], [1.9, 0, 0.4], [-0.9, 1.6, 0.4], [-0.9, -1.6, 0.4],
                                                  [0.3, 0.2, 5.5], [0.5, 0.1, 7.6]]),
}


def _mol(name, engine, oracle, basis="sto-3g"):
    if name == "h2o":
        return _h2o(engine, oracle, basis)
    sp, xyz = MOLS[name]
    return _pair(engine, oracle, sp, xyz, basis)


def test_boys_device_vs_mpmath(engine):
    import torch
    ref = json.load(open(os.path.join(GOLDEN, "boys_mpmath.json")))["values"]
    xs = sorted({x for _, x, _ in ref})
    F = engine.boys(torch.tensor(xs, dtype=torch.float64), 6).cpu().numpy()
    Ff = engine.boys(torch.tensor(xs, dtype=torch.float64), 6, fp32=True).cpu().numpy()
    for m, x, v in ref:
        i = xs.index(x)
        assert F[i, m] == pytest.approx(v, rel=2e-14, abs=1e-300), (m, x)
        assert Ff[i, m] == pytest.approx(v, rel=3e-6, abs=1e-37), (m, x)


def test_boys_trapezoid_device_vs_oracle(engine, oracle):
    import torch
    xs = [0.0, 5e-7, 1e-3, 0.7, 3.3, 17.0, 40.0]
    F = engine.boys(torch.tensor(xs, dtype=torch.float64), 4, mode="reference_trapezoid").cpu().numpy()
    for i, x in enumerate(xs):
        for m in range(5):
            assert F[i, m] == pytest.approx(oracle.boys(m, x, 1), rel=1e-13, abs=1e-300)


@pytest.mark.parametrize("name,basis", [("h2o", "sto-3g"), ("ch2o", "sto-6g"), ("nh3_co", "sto-2g")])
@pytest.mark.parametrize("mode", [0, 1])
def test_one_electron_vs_oracle(engine, oracle, name, basis, mode):
    em, om = _mol(name, engine, oracle, basis)
    with engine.System(em, boys_mode=mode) as s:
        S, T, V = (x.cpu().numpy() for x in s.one_electron())
    So, To, Vo = oracle.one_electron(om, boys_mode=mode)
    assert np.abs(S - So).max() < 1e-10
    assert np.abs(T - To).max() < 1e-10
    assert np.abs(V - Vo).max() < 1e-10


def test_one_electron_h2o_golden(engine, oracle):
    ref = json.load(open(os.path.join(GOLDEN, "h2o_sto3g.json")))
    em, om = _h2o(engine, oracle)
    with engine.System(em, boys_mode=1) as s:
        S, T, V = (x.cpu().numpy() for x in s.one_electron())
    assert np.abs(S - np.array(ref["S"])).max() < 1e-10
    assert np.abs(T - np.array(ref["T"])).max() < 1e-10
    assert np.abs(V - np.array(ref["V_trapezoid"])).max() < 1e-10


@pytest.mark.parametrize("name,basis", [("h2o", "sto-3g"), ("ch2o", "sto-3g"), ("nh3_co", "sto-4g")])
def test_eri_tensor_vs_oracle(engine, oracle, name, basis):
    em, om = _mol(name, engine, oracle, basis)
    with engine.System(em, schwarz_thresh=0.0) as s:
        eri = s.eri_tensor().cpu().numpy()
    ref = oracle.eri_tensor(om)
    assert np.abs(eri - ref).max() < 1e-12


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("mixed", 1e-7)])
def test_jk_vs_oracle(engine, oracle, precision, tol):
    import torch
    em, om = _mol("nh3_co", engine, oracle, "sto-3g")
    rng = np.random.default_rng(7)
    n = om.shells.nbf
    D = rng.standard_normal((n, n)) * 0.3
    D = D + D.T
    Db = rng.standard_normal((n, n)) * 0.3
    Db = Db + Db.T
    with engine.System(em, schwarz_thresh=1e-14) as s:
        J, K = s.jk(torch.tensor(D), precision=precision)
        J2, K2 = s.jk(torch.tensor(D + Db), torch.tensor(np.stack([D, Db])), precision=precision)
    Jo, Ko = oracle.jk(om, D, thresh=0)
    assert np.abs(J.cpu().numpy() - Jo).max() < tol
    assert np.abs(K.cpu().numpy() - Ko).max() < tol
    Jo2, _ = oracle.jk(om, D + Db, thresh=0)
    _, Kb = oracle.jk(om, Db, thresh=0)
    assert np.abs(J2.cpu().numpy() - Jo2).max() < tol
    assert np.abs(K2[0].cpu().numpy() - Ko).max() < tol
    assert np.abs(K2[1].cpu().numpy() - Kb).max() < tol


@pytest.mark.parametrize("name,basis,mode", [("h2o", "sto-3g", 0), ("h2o", "sto-3g", 1), ("ch2o", "sto-6g", 0),
                                             ("nh3_co", "sto-3g", 0)])
def test_scf_energy_vs_oracle(engine, oracle, name, basis, mode):
    em, om = _mol(name, engine, oracle, basis)
    r = engine.run(em, boys_mode=mode)
    ro = oracle.scf(om, boys_mode=mode)
    assert r.converged and ro.converged
    assert r.energy == pytest.approx(ro.energy, abs=1e-8)


def test_water_clusters_vs_oracle(engine, oracle):
    for f in ("h2o-2.xyz", "h2o-4.xyz"):
        n, c, s = oracle.read_xyz(os.path.join(MOL_DIR, f))
        em, om = _pair(engine, oracle, list(s), c.T)
        assert engine.run(em).energy == pytest.approx(oracle.scf(om).energy, abs=1e-8)


def test_uhf_vs_oracle(engine, oracle):
    em, om = _pair(engine, oracle, ["O", "H"], [[0, 0, 0], [0.1, 0, 1.83]])
    r = engine.run(em)
    ro = oracle.scf(om)
    assert r.uhf and ro.uhf
    assert r.energy == pytest.approx(ro.energy, abs=1e-8)
    # RHF == UHF for a closed shell
    em2, _ = _h2o(engine, oracle)
    assert engine.run(em2, scf_type="uhf").energy == pytest.approx(engine.run(em2).energy, abs=1e-9)


@pytest.mark.parametrize("name,basis", [("h2o", "sto-3g"), ("ch2o", "sto-3g")])
def test_gradient_vs_oracle(engine, oracle, name, basis):
    em, om = _mol(name, engine, oracle, basis)
    r = engine.run(em, gradient=True)
    ro = oracle.scf(om)
    go = oracle.gradient(om, ro)
    assert np.abs(r.gradient - go).max() < 1e-7
    assert np.abs(r.gradient.sum(0)).max() < 1e-8  # translational invariance


def test_uhf_gradient_vs_oracle(engine, oracle):
    em, om = _pair(engine, oracle, ["O", "H"], [[0, 0, 0], [0.1, 0, 1.83]])
    r = engine.run(em, gradient=True)
    go = oracle.gradient(om, oracle.scf(om))
    assert np.abs(r.gradient - go).max() < 1e-7


def test_gradient_vs_finite_differences_of_engine(engine):
    from pyfacc import geometry as G
    sp, xyz = G.alkane(3, seed=11)
    mol = engine.Molecule(sp, xyz)
    g = engine.run(mol, gradient=True).gradient
    h = 1e-4
    for a, x in [(0, 0), (1, 2), (5, 1)]:
        e = []
        for sgn in (1, -1):
            x2 = xyz.copy()
            x2[a, x] += sgn * h
            e.append(engine.run(engine.Molecule(sp, x2)).energy)
        assert g[a, x] == pytest.approx((e[0] - e[1]) / (2 * h), abs=2e-7)


def test_dropin_run_scf(engine, oracle, monkeypatch):
    import helper_functions as hf
    lib = hf.load_library()
    e = hf.run_scf(lib, "h2o.xyz", 1e-10, 50, ctypes.c_double(), "sto-3g")
    from pyfacc import _native as N
    assert N.lib().pyfacc_last_status() == N.OK
    em, om = _h2o(engine, oracle)
    assert e == pytest.approx(oracle.scf(om).energy, abs=1e-8)


def test_dropin_reports_missing_basis(engine):
    import helper_functions as hf
    from pyfacc import _native as N
    e = hf.run_scf(hf.load_library(), "h2o.xyz", 1e-10, 50, ctypes.c_double(), "sto-9g")
    assert np.isnan(e)
    assert N.lib().pyfacc_last_status() == N.ERR_BASIS_NOT_FOUND


def test_mixed_precision_delta_e(engine):
    from pyfacc import geometry as G
    sp, xyz = G.alkane(10, seed=1)
    mol = engine.Molecule(sp, xyz)
    e64 = engine.run(mol, gradient=True)
    emx = engine.run(mol, precision="mixed", gradient=True)
    assert emx.quartets["fp32"] > 0
    assert abs(emx.energy - e64.energy) <= 1e-6
    assert np.abs(emx.gradient - e64.gradient).max() <= 1e-5


@pytest.mark.parametrize("coarse_err", [0.0, 1e-3, 1e-1])
def test_mixed_coarse_phase(engine, coarse_err):
    """The all-FP32 builds of the first mixed iterations only shorten the
    way to the converged density: with the phase off (0), at its default
    and ended early, energy and gradient stay within the mixed-precision
    budget of FP64, and gradient FP32 splitting keeps translational
    invariance."""
    from pyfacc import geometry as G
    mol = engine.Molecule(*G.alkane(12, seed=3))
    e64 = engine.run(mol, gradient=True)
    emx = engine.run(mol, precision="mixed", gradient=True, coarse_err=coarse_err)
    assert emx.converged
    assert abs(emx.energy - e64.energy) <= 1e-6
    assert np.abs(emx.gradient - e64.gradient).max() <= 1e-5
    assert np.abs(emx.gradient.sum(0)).max() < 1e-8


def test_batch_mixed_coarse_phase(engine):
    from pyfacc import geometry as G
    clusters = G.water_clusters(count=6, seed=5)
    mols = [engine.Molecule(sp, xyz) for sp, xyz in clusters]
    ref = engine.run_batch(mols, gradient=True)
    for ce in (0.0, 1e-3):
        r = engine.run_batch(mols, gradient=True, precision="mixed", coarse_err=ce)
        for a, b in zip(r, ref):
            assert a.converged
            assert abs(a.energy - b.energy) <= 1e-6
            assert np.abs(a.gradient - b.gradient).max() <= 1e-5


def test_autograd_energy(engine):
    import torch
    em, _ = _h2o(engine, __import__("oracle"))
    c = torch.tensor(em.coords, requires_grad=True)
    E = engine.energy(c, em)
    E.backward()
    g = engine.run(em, gradient=True).gradient
    assert np.abs(c.grad.numpy() - g).max() < 1e-12
