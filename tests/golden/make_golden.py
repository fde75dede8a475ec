"""Regenerates the golden fixtures of tests/golden/.

* boys_mpmath.json -- F_m(x) from mpmath's 1F1 (independent of this repo):
  F_m(x) = 1F1(m+1/2; m+3/2; -x) / (2m+1)
* h2o_sto3g.json   -- the oracle's converged H2O/STO-3G energy (data/molecules/
  h2o.xyz) and its V matrix with the reference's trapezoid Boys function.
* c20h42_sto3g.json -- the oracle's converged energy and analytic gradient of
  the C20H42/STO-3G benchmark molecule (pyfacc.geometry.alkane(20, seed=1),
  142 basis functions); several minutes of CPU time, hence a fixture.
* c40h82_sto3g.json -- the same for C40H82/STO-3G (alkane(40, seed=40),
  282 basis functions), with the oracle's SCF iteration count; about half
  an hour on 8 cores.

    python tests/golden/make_golden.py [c20h42 | c40h82]
"""
import json
import os
import sys

import mpmath
import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def boys_values():
    mpmath.mp.dps = 40
    xs = [0.0, 1e-12, 1e-7, 1e-3, 0.05, 0.3, 1.0, 2.5, 5.0, 9.9, 14.0, 20.0, 27.5, 35.9, 36.1, 45.0, 80.0,
          250.0, 1e4, 1e6]
    out = []
    for m in range(0, 7):
        for x in xs:
            v = mpmath.hyp1f1(m + 0.5, m + 1.5, -x) / (2 * m + 1)
            out.append([m, x, float(v)])
    return out


def main():
    with open(os.path.join(HERE, "boys_mpmath.json"), "w") as fh:
        json.dump({"source": "mpmath.hyp1f1, 40 digits", "values": boys_values()}, fh, indent=0)
    import oracle as O
    n, c, s = O.read_xyz(os.path.join(ROOT, "pyfacc-scf_b200", "data", "molecules", "h2o.xyz"))
    mol = O.molecule(s, c.T, os.path.join(ROOT, "pyfacc-scf_b200", "data", "basis_set", "sto-3g.txt"))
    r = O.scf(mol)
    S, T, V = O.one_electron(mol, boys_mode=1)
    with open(os.path.join(HERE, "h2o_sto3g.json"), "w") as fh:
        json.dump({"source": "oracle, h2o.xyz, STO-3G, dE<1e-10, DIIS err<1e-8", "energy": r.energy,
                   "S": S.tolist(), "T": T.tolist(), "V_trapezoid": V.tolist()}, fh)


def alkane_fixture(n, seed):
    """The oracle's converged energy, analytic gradient, SCF iteration count
    and timings for alkane(n, seed) in STO-3G (core-Hamiltonian guess + DIIS,
    as oracle.scf runs it)."""
    import time
    import oracle as O
    sys.path.insert(0, os.path.join(ROOT, "pyfacc-scf_b200"))
    from pyfacc import geometry as G
    sp, xyz = G.alkane(n, seed=seed)
    mol = O.molecule(sp, xyz, os.path.join(ROOT, "pyfacc-scf_b200", "data", "basis_set", "sto-3g.txt"))
    t0 = time.perf_counter()
    r = O.scf(mol)
    t1 = time.perf_counter()
    g = O.gradient(mol, r)
    t2 = time.perf_counter()
    name = f"c{n}h{2 * n + 2}_sto3g.json"
    with open(os.path.join(HERE, name), "w") as fh:
        json.dump({"source": f"oracle, alkane({n}, seed={seed}), STO-3G RHF, dE<1e-10, DIIS err<1e-8, "
                             "Schwarz 1e-12",
                   "nbf": int(mol.shells.nbf), "energy": r.energy, "converged": bool(r.converged),
                   "scf_iterations": int(r.n_iter), "oracle_seconds": {"scf": t1 - t0, "gradient": t2 - t1},
                   "oracle_threads": os.cpu_count(),
                   "gradient": np.asarray(g).tolist()}, fh)


if __name__ == "__main__":
    if len(sys.argv) > 1 and sys.argv[1] == "c20h42":
        alkane_fixture(20, 1)
    elif len(sys.argv) > 1 and sys.argv[1] == "c40h82":
        alkane_fixture(40, 40)
    else:
        main()
