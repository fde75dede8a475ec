"""Host-injected failures that need no GPU: bad input is reported with a
status before any device work (the reference prints and carries on, or
aborts: la.f90:22-25,40-44, basis.f90:39).  Nothing here faults, traps or
hangs a device; the GPU-side cases (max_iter, coincident atoms) are in
test_gpu_failures.py."""
import ctypes
import math
import os

import numpy as np
import pytest


def _water():
    from pyfacc import geometry as G
    return G.water()


def _run_status(engine, mol, **opt):
    from pyfacc import _native as N
    m, keep = mol._struct()
    o = engine._options(**opt)
    r = N.Result()
    return N.lib().pyfacc_run(ctypes.byref(m), ctypes.byref(o), ctypes.byref(r))


@pytest.mark.parametrize("bad", [float("nan"), float("inf"), -float("inf")])
def test_non_finite_coordinates_are_invalid(engine, bad):
    from pyfacc import _native as N
    sp, xyz = _water()
    xyz = xyz.copy()
    xyz[1, 2] = bad
    assert _run_status(engine, engine.Molecule(sp, xyz)) == N.ERR_INVALID
    assert b"not finite" in N.lib().pyfacc_last_message()


def test_non_finite_coordinates_through_run_scf_c(engine):
    """The drop-in entry point keeps its void signature: NaN energy and the
    status for pyfacc_last_status()."""
    from pyfacc import _native as N
    L = N.lib()
    sp, xyz = _water()
    xyz = np.ascontiguousarray(xyz.copy())
    xyz[0, 0] = float("nan")
    species = (ctypes.c_char * 6)(*b"O H H ")
    z = np.array([8, 1, 1], dtype=np.int32)
    e = ctypes.c_double(0.0)
    L.run_scf_c(3, 10, 0, 5, 5, species, xyz.ctypes.data_as(N.P_double), 1e-10, 10, ctypes.byref(e), b"sto-3g",
                z.ctypes.data_as(N.P_int32))
    assert math.isnan(e.value)
    assert L.pyfacc_last_status() == N.ERR_INVALID


def test_unsupported_shell_type(engine, tmp_path):
    """A basis whose hydrogen section holds an F shell: the parser stops with
    UNSUPPORTED_L instead of misreading the block (basis.f90:76-82 has no
    branch for it and would read the exponent lines as shell headers)."""
    from pyfacc import _native as N
    d = tmp_path / "basis_set"
    d.mkdir()
    (d / "sto-3g.txt").write_text(
        "! a test basis in the Basis Set Exchange layout of data/basis_set/\n\n"
        "H     0\n"
        "S    3   1.00\n      0.3425250914D+01       0.1543289673D+00\n"
        "      0.6239137298D+00       0.5353281423D+00\n      0.1688554040D+00       0.4446345422D+00\n"
        "F    1   1.00\n      0.1000000000D+01       0.1000000000D+01\n"
        "****\n")
    mol = engine.Molecule(["H", "H"], [[0, 0, 0], [0, 0, 1.4]])
    assert _run_status(engine, mol, data_dir=str(tmp_path)) == N.ERR_UNSUPPORTED_L


def test_unknown_basis_and_element(engine):
    from pyfacc import _native as N
    mol = engine.Molecule(["H", "H"], [[0, 0, 0], [0, 0, 1.4]], basis="sto-9g")
    assert _run_status(engine, mol) == N.ERR_BASIS_NOT_FOUND
    m = engine.Molecule(["H", "H"], [[0, 0, 0], [0, 0, 1.4]])
    st, keep = m._struct()
    z = np.array([1, 1], dtype=np.int32)
    st.z = z.ctypes.data_as(N.P_int32)
    st.species = ctypes.cast(ctypes.create_string_buffer(b"XxH ", 4), ctypes.c_void_p)
    o = engine._options()
    assert N.lib().pyfacc_run(ctypes.byref(st), ctypes.byref(o), ctypes.byref(N.Result())) == N.ERR_ELEMENT


def test_inconsistent_spin_is_invalid(engine):
    """helper_functions.py:79-82 raises on an electron count that the
    multiplicity cannot hold; the engine reports INVALID."""
    from pyfacc import _native as N
    mol = engine.Molecule(["H", "H"], [[0, 0, 0], [0, 0, 1.4]], charge=1)
    # one electron, doublet: consistent; a charge of 3 leaves -1 electrons
    mol.charge = 3
    assert _run_status(engine, mol) == N.ERR_INVALID


@pytest.mark.parametrize("n", [-1, 65])
def test_diis_size_out_of_range_is_invalid(engine, n):
    """The Pulay subspace is read back with the energy every iteration into
    a fixed block of 64 overlaps: a larger (or negative) diis_size is
    refused before any device work."""
    from pyfacc import _native as N
    assert _run_status(engine, engine.Molecule(*_water()), diis_size=n) == N.ERR_INVALID
    assert b"diis_size" in N.lib().pyfacc_last_message()
