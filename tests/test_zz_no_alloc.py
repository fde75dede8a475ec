"""pyfacc_jk_noalloc -- J/K without any device allocation -- against the
ordinary handle-based J/K build, twice in a row.

The entry point exists for programs that give all of a GPU's memory to
their own allocator (a framework's caching allocator, a pool sized at
start-up), where a library's cudaMalloc would fail or fragment that pool.
This file is collected last so that a run stopping at the first failure has
already run every other test.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-10  # the J/K tolerance of the FP64 parity tests


def _molecule(engine):
    return engine.Molecule(["N", "H", "H", "H", "C", "O"],
                           [[0, 0, 0], [1.9, 0, 0.4], [-0.9, 1.6, 0.4], [-0.9, -1.6, 0.4], [0.3, 0.2, 5.5],
                            [0.5, 0.1, 7.6]], "sto-3g")


def test_noalloc_jk_matches_system_jk_twice(engine):
    import torch
    from pyfacc import _native as N
    mol = _molecule(engine)
    with engine.System(mol, schwarz_thresh=1e-12) as s:
        n = s.nbf
        rng = np.random.default_rng(3)
        D = rng.standard_normal((n, n)) * 0.3
        D = torch.tensor(D + D.T, device="cuda")
        J_ref, K_ref = s.jk(D)
    m, keep = mol._struct()
    data_dir = N.DATA_DIR.encode()
    outs = [(torch.empty(n, n, dtype=torch.float64, device="cuda"), torch.empty(n, n, dtype=torch.float64,
                                                                                 device="cuda")) for _ in range(2)]
    free = []
    for call, (J, K) in enumerate(outs):
        # stale values in the outputs must not leak into the result
        J.fill_(1e30)
        K.fill_(-1e30)
        torch.cuda.synchronize()
        free.append(torch.cuda.mem_get_info()[0])
        st = N.lib().pyfacc_jk_noalloc(ctypes.byref(m), data_dir, 1e-12, D.data_ptr(), J.data_ptr(), K.data_ptr())
        assert st == N.OK, N.lib().pyfacc_last_message()
        torch.cuda.synchronize()
        free.append(torch.cuda.mem_get_info()[0])
        assert (J - J_ref).abs().max().item() < TOL, call
        assert (K - K_ref).abs().max().item() < TOL, call
    # the first call may set the device up (module load, symbol lookup); the
    # second must not change the device's free memory at all
    assert free[3] == free[2], (free[2], free[3])


def test_noalloc_rejects_molecule_beyond_the_static_array(engine):
    import torch
    from pyfacc import _native as N
    from pyfacc import geometry as G
    sp, xyz = G.alkane(100, seed=4)
    mol = engine.Molecule(sp, xyz, "sto-3g")
    m, keep = mol._struct()
    d = torch.zeros(4, dtype=torch.float64, device="cuda")
    st = N.lib().pyfacc_jk_noalloc(ctypes.byref(m), N.DATA_DIR.encode(), 1e-12, d.data_ptr(), d.data_ptr(),
                                   d.data_ptr())
    assert st == N.ERR_INVALID
    assert b"scratch" in N.lib().pyfacc_last_message()
