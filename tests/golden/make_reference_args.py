"""Regenerates tests/golden/reference_driver_args.json from the reference's
own Python driver (src/python/helper_functions.py of PyFAcc-SCF), imported
from a checkout of the reference.

For every molecule file shipped in pyfacc-scf_b200/data/molecules the
reference's run_scf(lib, ...) is called with a stand-in `lib` whose
run_scf_c records the arguments it receives (the Fortran library is not
needed): natoms, nelectrons, charge, nalpha, nbeta, the species bytes, the
coordinates exactly as laid out in memory (hex of every double), eps_scf,
max_iter, the basis name and z_num.  Also compute_spin_electrons for a few
species lists, including the one the reference rejects.

    python tests/golden/make_reference_args.py /path/to/reference/checkout
"""
import ctypes
import json
import os
import struct
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


class Recorder:
    def __init__(self):
        self.calls = []

    def run_scf_c(self, natoms, nelectrons, charge, nalpha, nbeta, species, coords, eps, max_iter, energy, basis,
                  z_num):
        n = natoms.value
        xyz = [coords[i] for i in range(3 * n)]
        self.calls.append({
            "natoms": n, "nelectrons": nelectrons.value, "charge": charge.value, "nalpha": nalpha.value,
            "nbeta": nbeta.value, "species": bytes(species).decode("ascii"),
            "coords_hex": [struct.pack("<d", v).hex() for v in xyz], "eps_scf": eps.value,
            "max_iter": max_iter.value, "basis": basis.decode(), "z_num": [z_num[i] for i in range(n)]})


def main(ref):
    sys.path.insert(0, os.path.join(ref, "src", "python"))
    import helper_functions as H  # the reference's driver
    mol_dir = os.path.join(ROOT, "pyfacc-scf_b200", "data", "molecules")
    files = sorted(f for f in os.listdir(mol_dir) if f.endswith(".xyz"))
    out = {"source": "PyFAcc-SCF src/python/helper_functions.py run_scf / compute_spin_electrons", "calls": {}}
    cwd = os.getcwd()
    os.chdir(os.path.join(ROOT, "pyfacc-scf_b200"))  # read_xyz opens ./data/molecules/<file>
    try:
        for f in files:
            rec = Recorder()
            try:
                H.run_scf(rec, f, 1e-10, 10, ctypes.c_double(), "sto-3g")
                out["calls"][f] = rec.calls[0]
            except ValueError as e:
                out["calls"][f] = {"error": str(e)}
    finally:
        os.chdir(cwd)
    spins = {}
    for sp, charge in [(["H"], 0), (["H", "H"], 0), (["O", "O"], 0), (["N", "N"], 0), (["O", "H", "H"], 0),
                       (["O", "H", "H"], 1), (["C", "H", "H", "H"], 0), (["Li"], 0), (["O", "H"], -1)]:
        key = ",".join(sp) + f"/{charge}"
        try:
            spins[key] = list(H.compute_spin_electrons(np.array(sp), charge))
        except ValueError as e:
            spins[key] = {"error": str(e)}
    out["spin"] = spins
    with open(os.path.join(HERE, "reference_driver_args.json"), "w") as fh:
        json.dump(out, fh, indent=0)


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PYFACC_REFERENCE_DIR")
    if not ref:
        sys.exit("usage: make_reference_args.py <reference checkout> (or set PYFACC_REFERENCE_DIR)")
    main(ref)
