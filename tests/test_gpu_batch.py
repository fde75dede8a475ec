"""Batched engine (pyfacc_run_batch): many molecules of uneven size in the
same J/K launches and CUDA-graph SCF iterations, against the same molecules
run one by one (pyfacc_run) and against the oracle."""
import numpy as np
import pytest

from conftest import basis_file

pytestmark = pytest.mark.gpu


def _mols(engine, clusters, basis="sto-3g"):
    return [engine.Molecule(sp, xyz, basis) for sp, xyz in clusters]


def _small_set():
    from pyfacc import geometry as G
    out = [G.water()]
    out += G.water_clusters(count=5, seed=11, nmin=2, nmax=5)
    out.append(G.alkane(3, seed=7))
    return out


def test_batch_fp64_matches_single(engine):
    mols = _mols(engine, _small_set())
    rb = engine.run_batch(mols, gradient=True)
    for m, r in zip(mols, rb):
        rs = engine.run(m, gradient=True)
        assert r.converged and rs.converged
        assert r.energy == pytest.approx(rs.energy, abs=1e-8)
        assert np.abs(r.gradient - rs.gradient).max() < 1e-7
        assert np.abs(r.gradient.sum(0)).max() < 1e-8  # translational invariance


def test_batch_vs_oracle(engine, oracle):
    clusters = _small_set()[:3]
    rb = engine.run_batch(_mols(engine, clusters))
    for (sp, xyz), r in zip(clusters, rb):
        ro = oracle.scf(oracle.molecule(sp, xyz, basis_file()))
        assert r.energy == pytest.approx(ro.energy, abs=1e-8)


def test_batch_mixed_vs_fp64(engine):
    from pyfacc import geometry as G
    clusters = G.water_clusters(count=12, seed=3, nmin=4, nmax=9)
    mols = _mols(engine, clusters)
    r64 = engine.run_batch(mols, gradient=True)
    rmx = engine.run_batch(mols, gradient=True, precision="mixed")
    st = engine.batch_stats()
    assert st["quartets_fp32"] > 0
    for a, b in zip(r64, rmx):
        assert a.converged and b.converged
        assert abs(a.energy - b.energy) <= 1e-6
        assert np.abs(a.gradient - b.gradient).max() <= 1e-5


@pytest.mark.parametrize("width", [8, 16, 32])
def test_batch_task_widths_agree(engine, width):
    from pyfacc import geometry as G
    mols = _mols(engine, G.water_clusters(count=4, seed=5, nmin=3, nmax=6))
    ref = engine.run_batch(mols, task_width=32)
    r = engine.run_batch(mols, task_width=width)
    assert engine.batch_stats()["task_width"]["pp|pp"] == width
    for a, b in zip(ref, r):
        assert b.energy == pytest.approx(a.energy, abs=1e-10)


def test_single_molecule_task_widths_agree(engine):
    from pyfacc import geometry as G
    mol = engine.Molecule(*G.alkane(4, seed=2), "sto-3g")
    ref = engine.run(mol, gradient=True)
    for w in (8, 16):
        r = engine.run(mol, gradient=True, task_width=w)
        assert r.task_width == w
        assert r.energy == pytest.approx(ref.energy, abs=1e-10)
        assert np.abs(r.gradient - ref.gradient).max() < 1e-9


def test_batch_autotuner_picks_widths(engine):
    from pyfacc import geometry as G
    mols = _mols(engine, G.water_clusters(count=6, seed=8, nmin=3, nmax=7))
    r = engine.run_batch(mols, task_width=0)
    st = engine.batch_stats()
    assert set(st["task_width"].values()) <= {8, 16, 32}
    ref = engine.run_batch(mols, task_width=32)
    for a, b in zip(ref, r):
        assert b.energy == pytest.approx(a.energy, abs=1e-10)


def test_batch_mixes_open_shell_and_errors(engine):
    """Open-shell molecules leave the batch for the single-molecule path;
    a molecule with an unknown basis fails alone."""
    from pyfacc import geometry as G
    sp_r, xyz_r = G.radical(2, seed=5)
    mols = [engine.Molecule(*G.water(), "sto-3g"), engine.Molecule(sp_r, xyz_r, "sto-3g"),
            engine.Molecule(*G.alkane(2, seed=1), "sto-3g")]
    rb = engine.run_batch(mols, gradient=True)
    assert rb[1].uhf and not rb[0].uhf
    for m, r in zip(mols, rb):
        rs = engine.run(m, gradient=True)
        assert r.energy == pytest.approx(rs.energy, abs=1e-8)
    bad = engine.Molecule(*G.water(), "sto-9g")
    out = engine.run_batch([mols[0], bad], check=False)
    assert np.isfinite(out[0].energy) and np.isnan(out[1].energy)


def test_batch_repeat_is_reproducible(engine):
    from pyfacc import geometry as G
    mols = _mols(engine, G.water_clusters(count=8, seed=21, nmin=4, nmax=8))
    a = engine.run_batch(mols, precision="mixed", gradient=True)
    b = engine.run_batch(mols, precision="mixed", gradient=True)
    for x, y in zip(a, b):
        assert x.energy == pytest.approx(y.energy, abs=1e-9)
        assert x.n_iter == y.n_iter


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_s_only_molecules(engine, precision):
    """Molecules without p shells (H2, He2) leave the sp and pp classes of
    their segments empty; in a batch of only such molecules those task lists
    are empty altogether.  Both batches must match the one-by-one runs."""
    from pyfacc import geometry as G
    h2 = (["H", "H"], np.array([[0.0, 0.0, 0.0], [0.0, 0.0, 1.40]]))       # bohr
    he2 = (["He", "He"], np.array([[0.0, 0.0, 0.0], [0.0, 0.0, 5.6]]))
    h2b = (["H", "H"], np.array([[0.1, 0.0, 0.0], [0.0, 0.2, 1.45]]))
    for clusters in ([h2, he2, h2b], [h2, G.water(), he2]):
        mols = _mols(engine, clusters)
        rb = engine.run_batch(mols, gradient=True, precision=precision)
        for m, r in zip(mols, rb):
            rs = engine.run(m, gradient=True, precision=precision)
            assert r.converged and rs.converged
            assert r.energy == pytest.approx(rs.energy, abs=1e-7)
            assert np.abs(r.gradient - rs.gradient).max() < 1e-6


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_scf_is_one_graph_launch(engine, precision):
    """The whole batched SCF is one CUDA graph launch: the build variant of
    every iteration (all-FP32 coarse, full, incremental) and the loop's end
    are decided on the device; the results match the molecules run one by
    one."""
    from pyfacc import geometry as G
    mols = _mols(engine, G.water_clusters(count=12, seed=21, nmin=3, nmax=8))
    rb = engine.run_batch(mols, precision=precision)
    st = engine.batch_stats()
    assert st["scf_graph_launches"] == 1
    assert st["iterations"] >= 5
    for m, r in zip(mols[:4], rb[:4]):
        rs = engine.run(m, precision=precision)
        assert r.converged
        assert r.energy == pytest.approx(rs.energy, abs=1e-8 if precision == "fp64" else 1e-6)
