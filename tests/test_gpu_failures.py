"""Failures that need the device path: an SCF stopped by max_iter and an
overlap matrix made singular by coincident atoms.  Both are injected through
the input on the host; no kernel is made to fault or wait."""
import ctypes
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_max_iter_returns_last_energy_not_converged(engine):
    """rscf.f90:118-164 stops after max_iter and returns the last energy as
    if converged; the engine returns it too, with NOT_CONVERGED."""
    from pyfacc import _native as N
    from pyfacc import geometry as G
    mol = engine.Molecule(*G.water())
    r = engine.run(mol, max_iter=1, check=False)
    assert r.status == N.ERR_NOT_CONVERGED and not r.converged and r.n_iter == 1
    assert math.isfinite(r.energy)
    # (the first iteration's energy is that of the guess density, which need
    # not be idempotent, so it is not an upper bound of the converged one)
    full = engine.run(mol)
    assert full.converged and full.n_iter > 1
    # the drop-in entry point: the energy of the last iteration, status kept
    L = N.lib()
    sp, xyz = G.water()
    xyz = np.ascontiguousarray(xyz)
    e = ctypes.c_double(0.0)
    z = np.array([8, 1, 1], dtype=np.int32)
    L.run_scf_c(3, 10, 0, 5, 5, (ctypes.c_char * 6)(*b"O H H "), xyz.ctypes.data_as(N.P_double), 1e-10, 1,
                ctypes.byref(e), b"sto-3g", z.ctypes.data_as(N.P_int32))
    assert math.isfinite(e.value) and L.pyfacc_last_status() == N.ERR_NOT_CONVERGED


def test_coincident_atoms_are_linearly_dependent(engine):
    """Two hydrogens at the same point make two identical basis functions:
    la.f90:40-44 only warns about the zero overlap eigenvalue; here it is
    PYFACC_ERR_LINDEP, for one molecule and inside a batch."""
    from pyfacc import _native as N
    from pyfacc import geometry as G
    sp, xyz = G.water()
    mol = engine.Molecule(sp + ["H"], np.vstack([xyz, xyz[1]]))
    with pytest.raises(engine.PyfaccError) as ei:
        engine.run(mol)
    assert ei.value.status == N.ERR_LINDEP
    good = engine.Molecule(sp, xyz)
    rs = engine.run_batch([good, mol, good], check=False)
    assert rs[0].converged and rs[2].converged
    assert math.isnan(rs[1].energy) or not rs[1].converged
