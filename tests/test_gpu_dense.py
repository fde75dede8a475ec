"""The dense FP64 tensor-core products and the graph-driven TC2
purification of the SCF step (dense.cu) against torch's FP64 matmul and
eigh, through the C ABI.  These replace la.f90:7-57's dsyev-based density
step (rscf.f90:140-156); the SCF parity tests cover them end to end."""
import ctypes

import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12  # relative to the largest |C| (FP64 products, K <= 702)


@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (7, 7, 7), (16, 16, 16), (33, 33, 33), (142, 142, 142),
                                   (282, 282, 282), (30, 50, 20), (702, 702, 702)])
@pytest.mark.parametrize("ta,tb", [(0, 0), (0, 1), (1, 0), (1, 1)])
def test_dense_gemm_matches_torch(engine, m, n, k, ta, tb):
    import torch
    from pyfacc import _native as N
    g = torch.Generator(device="cuda").manual_seed(m * 1000 + n + 7 * k)
    A = torch.randn((k, m) if ta else (m, k), dtype=torch.float64, device="cuda", generator=g)
    B = torch.randn((n, k) if tb else (k, n), dtype=torch.float64, device="cuda", generator=g)
    C = torch.full((m, n), float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    assert N.lib().pyfacc_dense_gemm_dev(m, n, k, ta, A.data_ptr(), tb, B.data_ptr(), C.data_ptr(), 0, 0) == 0
    ref = (A.T if ta else A) @ (B.T if tb else B)
    assert torch.isfinite(C).all()
    assert ((C - ref).abs().max() / ref.abs().max().clamp_min(1e-300)).item() < TOL


@pytest.mark.parametrize("n", [5, 16, 47, 282])
def test_dense_gemm_symmetric_and_commutator(engine, n):
    import torch
    from pyfacc import _native as N
    g = torch.Generator(device="cuda").manual_seed(n)
    A = torch.randn((n, n), dtype=torch.float64, device="cuda", generator=g)
    S = A @ A.T
    C = torch.full((n, n), float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    # sym: A A^T from the upper triangle, mirrored
    assert N.lib().pyfacc_dense_gemm_dev(n, n, n, 0, A.data_ptr(), 1, A.data_ptr(), C.data_ptr(), 1, 0) == 0
    assert (C - C.T).abs().max().item() == 0.0
    assert ((C - S).abs().max() / S.abs().max()).item() < TOL
    # asym_a: (A - A^T) B
    B = torch.randn((n, n), dtype=torch.float64, device="cuda", generator=g)
    torch.cuda.synchronize()
    assert N.lib().pyfacc_dense_gemm_dev(n, n, n, 0, A.data_ptr(), 0, B.data_ptr(), C.data_ptr(), 0, 1) == 0
    ref = (A - A.T) @ B
    assert ((C - ref).abs().max() / ref.abs().max()).item() < TOL


@pytest.mark.parametrize("n,nocc", [(7, 5), (72, 31), (142, 81), (282, 161)])
def test_purify_is_the_occupied_projector(engine, n, nocc):
    import torch
    from pyfacc import _native as N
    g = torch.Generator(device="cuda").manual_seed(n + nocc)
    # a Fock-like spectrum: occupied levels below -0.2, virtual above +0.3
    Q, _ = torch.linalg.qr(torch.randn((n, n), dtype=torch.float64, device="cuda", generator=g))
    lev = torch.cat([-0.2 - 20 * torch.rand(nocc, dtype=torch.float64, device="cuda", generator=g),
                     0.3 + 5 * torch.rand(n - nocc, dtype=torch.float64, device="cuda", generator=g)])
    F = (Q * lev) @ Q.T
    F = 0.5 * (F + F.T)
    P = torch.full((n, n), float("nan"), dtype=torch.float64, device="cuda")
    steps = ctypes.c_int(0)
    torch.cuda.synchronize()
    assert N.lib().pyfacc_purify_dev(n, nocc, F.data_ptr(), P.data_ptr(), ctypes.byref(steps)) == 0
    w, V = torch.linalg.eigh(F)
    ref = V[:, :nocc] @ V[:, :nocc].T
    assert (P - ref).abs().max().item() < 1e-10
    assert abs(torch.trace(P).item() - nocc) < 1e-10
    assert 10 <= steps.value < 200
    # a degenerate level split by the occupation has no gap: reported, not faked
    lev2 = lev.clone()
    lev2[nocc - 1] = 0.0
    lev2[nocc] = 0.0
    F2 = (Q * lev2) @ Q.T
    F2 = 0.5 * (F2 + F2.T)
    torch.cuda.synchronize()
    st = N.lib().pyfacc_purify_dev(n, nocc, F2.data_ptr(), P.data_ptr(), ctypes.byref(steps))
    assert st in (N.OK, N.ERR_NOT_CONVERGED)
    if st == N.ERR_NOT_CONVERGED:
        assert steps.value >= 199
