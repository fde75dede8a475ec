"""Pins the large workloads against the oracle without a full oracle SCF.

A full SCF of the oracle at 211-702 basis functions takes hours of CPU time,
so these fixtures check the engine's converged FP64 density instead: one
oracle Fock build at that density gives the oracle's energy functional E[P]
and its commutator X^T (F P S - S P F) X.  A commutator below 1e-6 means the
density is the oracle's own SCF solution (to first order), and then E[P] is
the oracle's SCF energy to second order in the residual; the GPU tests
require the engine's energy to equal it to 1e-8 Ha.

Two steps, because the densities come from the GPU and the oracle runs on
the CPU:

    # on a machine with a B200: converged FP64 densities -> OUTDIR/<case>.npz
    python tests/golden/make_large_pins.py dump OUTDIR
    # on any machine (hours of CPU for all cases): fixtures pin_<case>.json
    python tests/golden/make_large_pins.py pin OUTDIR [case ...]

Cases: C30H61 STO-6G UHF (pyfacc.geometry.radical(30, seed=2)), C40H82 and
C100H202 STO-3G RHF (alkane(40, seed=40), alkane(100, seed=4)) and the
reference's data/molecules/rna1.xyz in STO-3G.  With ``--gradient`` the pin
step also evaluates the oracle's analytic gradient at the engine's density
(P and W = 1/2 P F P per spin, from the oracle's F).
"""
from __future__ import annotations

import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
PKG = os.path.join(ROOT, "pyfacc-scf_b200")
for _p in (PKG, os.path.join(ROOT, "oracle")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

CASES = {
    "c30h61_sto6g_uhf": "C30H61 radical, STO-6G UHF doublet (211 bf), radical(30, seed=2)",
    "c40h82_sto3g": "C40H82, STO-3G RHF (282 bf), alkane(40, seed=40)",
    "c100h202_sto3g": "C100H202, STO-3G RHF (702 bf), alkane(100, seed=4)",
    "rna1_sto3g": "data/molecules/rna1.xyz, STO-3G RHF (491 bf)",
}


def case_geometry(name):
    """species, bohr coordinates (natoms, 3), basis name of a case."""
    from pyfacc import geometry as G
    if name == "c30h61_sto6g_uhf":
        sp, xyz = G.radical(30, seed=2)
        return sp, xyz, "sto-6g"
    if name == "c40h82_sto3g":
        sp, xyz = G.alkane(40, seed=40)
        return sp, xyz, "sto-3g"
    if name == "c100h202_sto3g":
        sp, xyz = G.alkane(100, seed=4)
        return sp, xyz, "sto-3g"
    if name == "rna1_sto3g":
        import pyfacc
        m = pyfacc.Molecule.from_xyz(os.path.join(PKG, "data", "molecules", "rna1.xyz"), "sto-3g")
        return list(m.species), m.coords, "sto-3g"
    raise KeyError(name)


def dump(outdir, names):
    import ctypes
    import torch
    import pyfacc
    from pyfacc import _native as N
    os.makedirs(outdir, exist_ok=True)
    for name in names:
        sp, xyz, basis = case_geometry(name)
        mol = pyfacc.Molecule(sp, xyz, basis)
        with pyfacc.System(mol, precision="fp64", max_iter=200) as s:
            r = s.scf(matrices=True)
            g = s.gradient()
            n = s.nbf
            P = r.matrices["P"]
            out = dict(species=np.array(sp), xyz=np.asarray(xyz), basis=basis, P=P, energy=r.energy,
                       n_iter=r.n_iter, converged=r.converged, uhf=r.uhf, gradient=g,
                       last_diis_error=r.last_diis_error)
            if r.uhf:  # the engine's device density is the alpha density for UHF
                from pyfacc.distributed import _CudaView
                ptr = ctypes.c_void_p()
                N.check(N.lib().pyfacc_system_density_dev(s.handle, ctypes.byref(ptr)), "pyfacc_system_density_dev")
                Pa = torch.as_tensor(_CudaView(int(ptr.value), n * n), device="cuda")
                out["Pa"] = Pa.cpu().numpy().reshape(n, n).copy()
        np.savez_compressed(os.path.join(outdir, f"{name}.npz"), **out)
        print(f"{name}: nbf {n}, E = {r.energy:.10f}, {r.n_iter} iterations, converged {r.converged}", flush=True)


def pin(outdir, names, with_gradient=False):
    import oracle as O
    for name in names:
        d = np.load(os.path.join(outdir, f"{name}.npz"))
        sp, xyz, basis = case_geometry(name)
        assert np.array_equal(np.asarray(xyz), d["xyz"]), f"{name}: geometry differs from the dump"
        mol = O.molecule(list(sp), np.asarray(xyz), os.path.join(PKG, "data", "basis_set", f"{basis}.txt"))
        uhf = bool(d["uhf"])
        P = np.ascontiguousarray(d["P"])
        t0 = time.perf_counter()
        S, T, V = O.one_electron(mol)
        H = T + V
        t1 = time.perf_counter()
        if uhf:
            Pa = np.ascontiguousarray(d["Pa"])
            Ds = [Pa, P - Pa]
            J, K = O.jk(mol, np.stack(Ds), 1e-12)
            Jt = J[0] + J[1]
            Fs = [H + Jt - K[0], H + Jt - K[1]]
            E = 0.5 * (np.sum(P * H) + np.sum(Ds[0] * Fs[0]) + np.sum(Ds[1] * Fs[1]))
            pairs = list(zip(Fs, Ds))
        else:
            J, K = O.jk(mol, P, 1e-12)
            Fs = [H + J - 0.5 * K]
            E = 0.5 * np.sum(P * (H + Fs[0]))
            pairs = [(Fs[0], P)]
        t2 = time.perf_counter()
        s, U = np.linalg.eigh(S)
        X = U / np.sqrt(s)
        comm = max(float(np.abs(X.T @ (F @ D @ S - S @ D @ F) @ X).max()) for F, D in pairs)
        en = O.enuc(mol)
        nocc = [mol.nalpha, mol.nbeta] if uhf else [(mol.nalpha + mol.nbeta + 1) // 2]
        tr = [float(np.sum(D * S)) for _, D in pairs]
        rec = {
            "case": CASES[name],
            "generator": "tests/golden/make_large_pins.py (dump on a B200, pin with the oracle on the CPU)",
            "nbf": int(mol.shells.nbf), "natoms": int(mol.natoms), "basis": basis, "uhf": uhf,
            "oracle_energy_at_engine_density": float(E + en),
            "oracle_e_nuc": float(en),
            "oracle_commutator_max": comm,
            "electron_count_tr_PS": tr, "occupations": nocc,
            "engine_fp64_energy_at_dump": float(d["energy"]),
            "engine_scf_iterations_at_dump": int(d["n_iter"]),
            "engine_last_diis_error_at_dump": float(d["last_diis_error"]),
            "oracle_seconds": {"one_electron": t1 - t0, "fock_build": t2 - t1},
            "oracle_threads": os.cpu_count(),
        }
        if with_gradient:
            # W per spin = P_s F_s P_s (UHF), 1/2 P F P for the RHF total density
            if uhf:
                W = Ds[0] @ Fs[0] @ Ds[0] + Ds[1] @ Fs[1] @ Ds[1]
                res = O.ScfResult(E + en, E, en, True, 0, True, None, None, Ds, P, S, H, [])
            else:
                W = 0.5 * P @ Fs[0] @ P
                res = O.ScfResult(E + en, E, en, True, 0, False, None, None, [0.5 * P, 0.5 * P], P, S, H, [])
            t3 = time.perf_counter()
            g = gradient_with_w(O, mol, res, W)
            rec["oracle_gradient_at_engine_density"] = np.asarray(g).tolist()
            rec["engine_fp64_gradient_at_dump"] = np.asarray(d["gradient"]).tolist()
            rec["oracle_seconds"]["gradient"] = time.perf_counter() - t3
        path = os.path.join(HERE, f"pin_{name}.json")
        with open(path, "w") as fh:
            json.dump(rec, fh, indent=1)
        print(f"{name}: oracle E[P] = {E + en:.10f} (engine {float(d['energy']):.10f}, "
              f"diff {E + en - float(d['energy']):.2e}), commutator {comm:.2e}, "
              f"{t2 - t0:.0f} s", flush=True)


def gradient_with_w(O, mol, res, W):
    """The oracle's analytic gradient with a given energy-weighted density."""
    na = mol.natoms
    g = [np.zeros((na, 3)) for _ in range(4)]
    O.lib().orc_gradient(*mol.shells.args(), na, O._ptr(mol.xyz), O._ptr(mol.Z), 0,
                         O._ptr(np.ascontiguousarray(res.P)), O._ptr(np.ascontiguousarray(res.D[0])),
                         O._ptr(np.ascontiguousarray(res.D[1])), O._ptr(np.ascontiguousarray(W)), 1e-12,
                         *[O._ptr(x) for x in g])
    return g[0] + g[1] + g[2] + g[3]


def main(argv):
    if len(argv) < 2 or argv[0] not in ("dump", "pin"):
        print(__doc__)
        return 2
    mode, outdir = argv[0], argv[1]
    rest = [a for a in argv[2:] if not a.startswith("--")]
    names = rest or list(CASES)
    if mode == "dump":
        dump(outdir, names)
    else:
        pin(outdir, names, with_gradient="--gradient" in argv)
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv[1:]))
