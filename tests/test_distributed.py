"""Sharded Fock builds: partition + reduction over a world_size-2 process
group on CPU (gloo), and the engine's sharded SCF + gradient on one GPU with
two host-thread shards joined by a host-side sum (no kernel waits on
another)."""
import os
import threading

import numpy as np
import pytest

from conftest import MOL_DIR, PKG, basis_file


def test_partition_covers_every_item_once(engine):
    from pyfacc.distributed import partition
    rng = np.random.default_rng(2)
    for n, parts in [(10, 2), (100, 4), (37, 8), (5, 8)]:
        c = rng.uniform(0.1, 5.0, n)
        b = partition(c, parts)
        assert b[0] == 0 and b[-1] == n and all(x <= y for x, y in zip(b, b[1:]))
        if n >= 4 * parts:
            shares = np.array([c[b[k]:b[k + 1]].sum() for k in range(parts)])
            assert shares.max() <= c.sum() / parts + c.max() + 1e-12


def _worker(rank, world, port, out_dir):
    import sys
    sys.path.insert(0, PKG)
    sys.path.insert(0, os.path.join(os.path.dirname(PKG), "oracle"))
    import torch
    import torch.distributed as dist
    import oracle as O
    from pyfacc.distributed import partition, allreduce_sum
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    n, c, s = O.read_xyz(os.path.join(MOL_DIR, "h2o-2.xyz"))
    mol = O.molecule(list(s), c.T, basis_file())
    ns = len(mol.shells.l)
    npair = ns * (ns + 1) // 2
    rng = np.random.default_rng(9)
    D = rng.standard_normal((mol.shells.nbf,) * 2)
    D = D + D.T
    b = partition(np.arange(1, npair + 1, dtype=float), world)  # bra pair ij has ij+1 kets
    J, K = O.jk_range(mol, D, b[rank], b[rank + 1])
    t = torch.tensor(np.stack([J, K]))
    allreduce_sum(t)
    if rank == 0:
        Jf, Kf = O.jk(mol, D)
        np.save(os.path.join(out_dir, "err.npy"),
                np.array([np.abs(t[0].numpy() - Jf).max(), np.abs(t[1].numpy() - Kf).max()]))
    dist.barrier()
    dist.destroy_process_group()


def test_sharded_jk_gloo_world2(tmp_path, oracle):
    import socket
    import torch.multiprocessing as mp
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    mp.start_processes(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    err = np.load(tmp_path / "err.npy")
    assert err.max() < 1e-12


class _HostSum:
    """Reducer for shards in threads of one process: every shard hands in its
    device buffer, the host sums the copies and writes the sum back."""

    def __init__(self, n):
        self.n = n
        self.bar = threading.Barrier(n, timeout=120)
        self.lock = threading.Lock()
        self.parts = {}

    def make(self, rank):
        from pyfacc import _native as N

        def fn(ctx, ptr, count):
            import torch
            from pyfacc.distributed import _CudaView
            t = torch.as_tensor(_CudaView(int(ptr), int(count)), device="cuda")
            with self.lock:
                self.parts[rank] = t.cpu()
            self.bar.wait()
            total = sum(self.parts[r] for r in range(self.n))
            self.bar.wait()
            t.copy_(total.to("cuda"))
            torch.cuda.synchronize()
            return 0

        return N.REDUCE_FN(fn)


@pytest.mark.gpu
def test_sharded_scf_two_shards_one_gpu(engine):
    from pyfacc import geometry as G
    from pyfacc.distributed import attach_reducer
    sp, xyz = G.alkane(6, seed=3)
    mol = engine.Molecule(sp, xyz, "sto-3g")
    ref = engine.run(mol, gradient=True)
    hs = _HostSum(2)
    results = {}

    def shard(rank):
        s = engine.System(mol, shard_rank=rank, shard_count=2)

        class R:
            cb = hs.make(rank)
        attach_reducer(s, R())
        r = s.scf()
        results[rank] = (r.energy, s.gradient(), r.quartets["fp64"])
        s.close()

    th = [threading.Thread(target=shard, args=(r,)) for r in range(2)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    for rank in range(2):
        e, g, q = results[rank]
        assert e == pytest.approx(ref.energy, abs=1e-9)
        assert np.abs(g - ref.gradient).max() < 1e-8
    # each shard evaluated a share of the quartets
    assert 0 < results[0][2] < ref.quartets["fp64"] and 0 < results[1][2] < ref.quartets["fp64"]


def _sharded_worker(rank, world, port, out_dir, precision):
    """One rank of the product's sharded path: pyfacc.distributed.
    sharded_system (its TorchReducer all-reduces every partial J/K and the
    two-electron gradient over the process group), SCF + gradient."""
    import sys
    sys.path.insert(0, PKG)
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    import pyfacc
    from pyfacc import geometry as G
    from pyfacc.distributed import sharded_system
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    sp, xyz = G.alkane(8, seed=5)
    mol = pyfacc.Molecule(sp, xyz, "sto-3g")
    s = sharded_system(mol, precision=precision)
    r = s.scf()
    g = s.gradient()
    np.save(os.path.join(out_dir, f"rank{rank}.npy"),
            np.concatenate([[r.energy, float(r.converged), float(r.quartets["fp64"] + r.quartets["fp32"])],
                            g.ravel()]))
    s.close()
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_sharded_system_two_processes_gloo(engine, tmp_path, precision):
    """Two processes share one GPU and one molecule through the product's
    torch.distributed reducer (gloo all-reduces the CUDA buffers on the host
    side; no kernel of one rank waits on the other): both ranks reproduce
    the unsharded energy and gradient."""
    import socket
    import torch.multiprocessing as mp
    from pyfacc import geometry as G
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    mp.start_processes(_sharded_worker, args=(2, port, str(tmp_path), precision), nprocs=2, join=True,
                       start_method="spawn")
    sp, xyz = G.alkane(8, seed=5)
    ref = engine.run(engine.Molecule(sp, xyz, "sto-3g"), gradient=True, precision=precision)
    nq_ref = ref.quartets["fp64"] + ref.quartets["fp32"]
    for rank in range(2):
        v = np.load(tmp_path / f"rank{rank}.npy")
        e, conv, nq, g = v[0], v[1], v[2], v[3:].reshape(-1, 3)
        assert conv == 1.0
        tol_e, tol_g = (1e-9, 1e-8) if precision == "fp64" else (1e-6, 1e-5)
        assert e == pytest.approx(ref.energy, abs=tol_e)
        assert np.abs(g - ref.gradient).max() < tol_g
        if precision == "fp64":
            assert 0 < nq < nq_ref  # each rank evaluated a share of the same static lists
